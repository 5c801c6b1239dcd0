"""Restart through the scripting surface: LsmMpi.createRestartCheckPointer writes the
reference's checkpoint files (master info + worker file) during run(), and a restart script
(groups from the script, state from LsmMpi.loadCheckPoint) continues the run.  Snapshots
(createCheckPointer) write the visualisation format.  Needs a GPU.

Bar: the restarted run follows the uninterrupted one to within the file's 12 significant
digits (positions within 1e-8 of their scale after 60 more steps).
"""
import os

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

DT, NSTEPS, SPLIT = 1e-5, 120, 60


def _lattice():
    rng = np.random.default_rng(11)
    g = np.stack(np.meshgrid(np.arange(4), np.arange(5), np.arange(4), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) + rng.uniform(-0.01, 0.01, size=g.shape)
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1)
    np.fill_diagonal(d, np.inf)
    rad = np.full(len(g), 0.495)
    i1, i2 = np.nonzero(np.triu(d - 2 * 0.495 <= 0.02, 1))
    vel = rng.normal(0, 0.05, size=(len(g), 3))
    return pos, rad, [(1, int(a), int(b)) for a, b in zip(i1, i2)], vel


class Loader:
    def __init__(self, sim):
        self.sim = sim

    def run(self):
        from esys.lsm.util import Vec3

        self.sim.moveWallBy("bottom", Vec3(0, 2e-4, 0))
        self.sim.moveWallBy("top", Vec3(0, -2e-4, 0))


def _script(restart_from=None, checkpoint_prefix=None, snapshot_prefix=None, nsteps=NSTEPS):
    from esys.lsm import (LinDampingPrms, LsmMpi, NRotElasticWallPrms, RestartCheckPointPrms, CheckPointPrms,
                          RotBondPrms, RotDampingPrms, RotFrictionPrms, RotSphere, Runnable)
    from esys.lsm.util import BoundingBox, Vec3

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1])
    sim.initNeighbourSearch("RotSphere", 1.25, 0.2)
    sim.setTimeStepSize(DT)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 5, 4)))
    if restart_from is None:
        pos, rad, conns, vel = _lattice()
        parts = []
        for k in range(len(pos)):
            p = RotSphere(k, Vec3(*pos[k]), float(rad[k]), float(S.sphere_mass(rad[k])))
            p.setLinearVelocity(Vec3(*vel[k]))
            parts.append(p)
        sim.createParticles(parts)
        sim.createConnections(conns)
    sim.createInteractionGroup(RotBondPrms("bonds", 1e5, 1e5, 1e3, 1e3, 5.0, 5.0, 5.0, 5.0, 1))
    sim.createInteractionGroup(RotFrictionPrms("friction", 1e5, 0.6, 0.6, 1e5))
    sim.createExclusion("bonds", "friction")
    if restart_from is None:
        sim.createWall("bottom", Vec3(0, 0.0, 0), Vec3(0, 1, 0))
        sim.createWall("top", Vec3(0, 5.0, 0), Vec3(0, -1, 0))
    else:
        sim.loadCheckPoint(restart_from)
    sim.createInteractionGroup(NRotElasticWallPrms("bottom_w", "bottom", 1e5))
    sim.createInteractionGroup(NRotElasticWallPrms("top_w", "top", 1e5))
    sim.createInteractionGroup(LinDampingPrms("damp", 0.01, 50))
    sim.createInteractionGroup(RotDampingPrms("rdamp", 0.01, 50))

    class L(Runnable):
        def __init__(self):
            Runnable.__init__(self)
            self.l = Loader(sim)

        def run(self):
            self.l.run()

    sim.addPreTimeStepRunnable(L())
    if checkpoint_prefix:
        sim.createRestartCheckPointer(RestartCheckPointPrms(checkpoint_prefix, 0, nsteps, SPLIT))
    if snapshot_prefix:
        sim.createCheckPointer(CheckPointPrms(snapshot_prefix, 0, nsteps, SPLIT))
    sim.setNumTimeSteps(nsteps)
    sim.run()
    return sim


def _state(sim):
    s = sim._sim
    p = s.particles()
    o = np.argsort(p["id"])
    return {k: p[k][o] for k in ("id", "pos", "vel", "angvel", "quat")}


def test_restart_continues_the_run(dem_lib, tmp_path):
    prefix = str(tmp_path / "cp")
    full = _script(checkpoint_prefix=prefix, snapshot_prefix=str(tmp_path / "snap"))
    for t in (0, SPLIT, NSTEPS):
        assert os.path.exists(f"{prefix}_t={t}_0.txt") and os.path.exists(f"{prefix}_t={t}_1.txt"), t
    info = open(f"{prefix}_t={SPLIT}_0.txt").read().split("\n")
    assert info[0] == "V 3" and info[3] == str(SPLIT) and info[-1].endswith(f"cp_t={SPLIT}_1.txt")
    cp = S.parse_checkpoint(f"{prefix}_t={SPLIT}_1.txt")
    assert len(cp["particles"]) == 80 and len(cp["bonds"]) > 0 and set(cp["walls"]) == {"bottom", "top"}
    # snapshot worker file: the particle count, one record per particle (22 + 7 fields), the bond records
    snap = open(str(tmp_path / "snap") + f"_t={SPLIT}_1.txt").read().split("\n")
    assert int(snap[0]) == 80 and len(snap[1].split()) == 29
    restarted = _script(restart_from=f"{prefix}_t={SPLIT}_0.txt")
    assert restarted.getTimeStep() == NSTEPS
    a, b = _state(full), _state(restarted)
    assert np.array_equal(a["id"], b["id"])
    assert np.abs(a["pos"] - b["pos"]).max() <= 1e-8 * np.abs(a["pos"]).max()
    assert np.abs(a["vel"] - b["vel"]).max() <= 1e-6 * max(np.abs(a["vel"]).max(), 1e-12)
    full.exit()
    restarted.exit()
