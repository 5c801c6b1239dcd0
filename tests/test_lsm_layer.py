"""The esys.lsm scripting surface (LsmMpi, *Prms, particles, runnables): host
logic checked on the CPU by running a reference-style script on the CPU
oracle backend and comparing with the same calls made directly."""
import numpy as np

import scenarios as S


class OrcBackend:
    """Adapts the oracle's ctypes front end to the DemSim methods LsmMpi uses."""

    def __new__(cls, *a):
        import oracle

        sim = oracle.OracleSim("orc", *a)
        sim.set_timestep = lambda dt: None
        sim.num_particles = lambda: len(sim.particles()["id"])
        sim.close = lambda: None
        return sim


def test_lsmmpi_gravity_script_matches_direct_calls(oracle_libs):
    from esys.lsm import (GravityPrms, LinDampingPrms, LsmMpi, NRotElasticPrms, NRotElasticWallPrms, NRotSphere,
                          Runnable)
    from esys.lsm.util import BoundingBox, Vec3

    class Loader(Runnable):
        def __init__(self, sim):
            Runnable.__init__(self)
            self.sim, self.n = sim, 0

        def run(self):
            self.sim.moveWallBy("floor", Vec3(0, 0, 1e-4))
            self.n += 1

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=OrcBackend)
    sim.initNeighbourSearch(particleType="NRotSphere", gridSpacing=1.2, verletDist=0.2)
    sim.setNumTimeSteps(60)
    sim.setTimeStepSize(1e-4)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 8)))
    rng = np.random.default_rng(7)
    parts = []
    for i in range(12):
        p = NRotSphere(id=i, posn=Vec3(0.6 + (i % 3) * 1.1, 0.6 + (i // 3 % 2) * 1.1, 0.6 + (i // 6) * 1.0),
                       radius=0.45, mass=float(S.sphere_mass(0.45)))
        p.setLinearVelocity(Vec3(*rng.normal(0, 0.5, 3)))
        parts.append(p)
    sim.createParticles(parts)
    sim.createInteractionGroup(NRotElasticPrms(name="elastic", normalK=1000.0))
    sim.createInteractionGroup(GravityPrms(name="g", acceleration=Vec3(0, 0, -9.81)))
    sim.createWall(name="floor", posn=Vec3(0, 0, 0), normal=Vec3(0, 0, 1))
    sim.createInteractionGroup(NRotElasticWallPrms(name="floor_w", wallName="floor", normalK=1000.0))
    sim.createInteractionGroup(LinDampingPrms(name="damp", viscosity=0.01, maxIterations=100))
    loader = Loader(sim)
    sim.addPreTimeStepRunnable(loader)
    sim.run()
    assert loader.n == 60 and sim.getTimeStep() == 60

    d = OrcBackend("NRotSphere", 1.2, 0.2, (0, 0, 0), (4, 4, 8), (0, 0, 0), 1e-4)
    d.add_particles([p.getId() for p in parts], [list(p.getPosn()) for p in parts], [0.45] * 12,
                    [float(S.sphere_mass(0.45))] * 12, tag=[0] * 12, vel=[list(p.getLinearVelocity()) for p in parts])
    d.add_elastic_group("elastic", 1000.0, True)
    d.add_gravity("g", (0, 0, -9.81))
    d.add_wall("floor", (0, 0, 0), (0, 0, 1))
    d.add_wall_group("floor_w", "floor", 1000.0)
    d.add_damping(0, 0.01, 100)
    for _ in range(60):
        d.move_wall("floor", (0, 0, 1e-4))
        d.step(1)
    a, b = sim._sim.particles(), d.particles()
    for k in ("pos", "vel", "force"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(np.array(list(sim.getWallForce("floor"))), d.wall("floor")[1])
    assert len(sim.getParticleList()) == 12


def test_lsmmpi_rejects_groups_outside_the_path(oracle_libs):
    import pytest

    from esys.lsm import LsmMpi
    from esys.lsm.util import BoundingBox, Vec3

    sim = LsmMpi(_backend=OrcBackend)
    with pytest.raises(NotImplementedError):
        sim.initNeighbourSearch(particleType="RotThermSphere", gridSpacing=1.0, verletDist=0.1)
    sim.initNeighbourSearch(particleType="RotSphere", gridSpacing=1.0, verletDist=0.1)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(3, 3, 3)))
    with pytest.raises(NotImplementedError):
        sim.readMesh("x.msh", "mesh")


def test_connection_finder_bonds_touching_pairs():
    from esys.lsm import ConnectionFinder, RotSphere
    from esys.lsm.util import Vec3

    ps = [RotSphere(0, Vec3(0, 0, 0), 0.5, 1.0), RotSphere(1, Vec3(1.0005, 0, 0), 0.5, 1.0),
          RotSphere(2, Vec3(3, 0, 0), 0.5, 1.0)]
    c = list(ConnectionFinder(maxDist=1e-3, bondTag=4, pList=ps))
    assert c == [(4, 0, 1)]


class RefBackend(OrcBackend):
    """The reference-built harness behind the same adapter."""

    def __new__(cls, *a):
        import oracle

        sim = oracle.OracleSim("ref", *a)
        sim.set_timestep = lambda dt: None
        sim.num_particles = lambda: len(sim.particles()["id"])
        sim.close = lambda: None
        return sim


def test_lsmmpi_widened_law_prms_match_direct_calls(oracle_libs):
    """HertzMindlinPrms, NRotFrictionPrms, LocalDampingPrms and the older createDamping /
    createGravity spellings reach the same groups (time step included: LsmMpiPy's
    createHertzMindlinIG and createNRotFrictionInteractGrp take it from the model) as direct calls."""
    import pytest

    from esys.lsm import (GravityPrms, HertzMindlinPrms, HertzMindlinViscoPrms, LocalDampingPrms, LsmMpi,
                          NRotFrictionPrms, NRotSphere)
    from esys.lsm.util import BoundingBox, Vec3

    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    for law in ("hm", "hmv", "nfric"):
        sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=RefBackend)
        sim.initNeighbourSearch(particleType="NRotSphere", gridSpacing=1.2, verletDist=0.1)
        sim.setNumTimeSteps(80)
        sim.setTimeStepSize(1e-4)
        sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 8)))
        rng = np.random.default_rng(11)
        parts = []
        for i in range(18):
            p = NRotSphere(id=i, posn=Vec3(0.6 + (i % 3) * 0.9, 0.6 + (i // 3 % 2) * 0.9, 0.6 + (i // 6) * 0.9),
                           radius=0.47, mass=float(S.sphere_mass(0.47)))
            p.setLinearVelocity(Vec3(*rng.normal(0, 0.5, 3)))
            parts.append(p)
        sim.createParticles(parts)
        if law == "hm":
            sim.createInteractionGroup(HertzMindlinPrms(name="c", youngsModulus=1e4, poissonsRatio=0.3,
                                                        dynamicMu=0.4))
        elif law == "hmv":
            sim.createInteractionGroup(HertzMindlinViscoPrms(name="c", youngsModulus=1e4, poissonsRatio=0.3,
                                                             dynamicMu=0.4, restitution=0.7))
        else:
            sim.createInteractionGroup(NRotFrictionPrms(name="c", normalK=1e4, dynamicMu=0.4, shearK=5e3))
        sim.createGravity(GravityPrms(name="g", acceleration=Vec3(0, 0, -9.81)))
        sim.createDamping(LocalDampingPrms(name="local", viscosity=0.05))
        sim.run()

        d = RefBackend("NRotSphere", 1.2, 0.1, (0, 0, 0), (4, 4, 8), (0, 0, 0), 1e-4)
        d.add_particles([p.getId() for p in parts], [list(p.getPosn()) for p in parts], [0.47] * 18,
                        [float(S.sphere_mass(0.47))] * 18, tag=[0] * 18,
                        vel=[list(p.getLinearVelocity()) for p in parts])
        if law == "hm":
            d.add_hertz_mindlin_group("c", 1e4, 0.3, 0.4, 1e-4)
        elif law == "hmv":
            d.add_hertz_mindlin_visco_group("c", 1e4, 0.3, 0.4, 0.7, 1e-4)
        else:
            d.add_nrot_friction_group("c", 1e4, 0.4, 5e3, 1e-4, True)
        d.add_gravity("g", (0, 0, -9.81))
        d.add_local_damping("local", 0, 0.05)
        d.step(80)
        a, b = sim._sim.particles(), d.particles()
        for k in ("pos", "vel", "force"):
            assert np.array_equal(a[k], b[k]), (law, k)
        if law != "hmv":  # the harness lists the pairs of the other two laws
            st = np.array(d.pairs("c")[2])
            assert st[:, 4].sum() > 5, law  # contacts were touching
        else:
            assert np.abs(b["force"]).max() > 0


import pytest as _pytest


@_pytest.mark.parametrize("law", ["dzc", "sc"])
def test_lsmmpi_brittle_beam_prms_match_direct_calls(oracle_libs, law):
    """BrittleBeamDZCPrms(name, E, nu, cohesion, frictionAngle, tensileCutoff, compressCutoff, beta1,
    beta2, tag) reaches the group the raw-stiffness call makes (ARotBondedIGP's kr = kb = pi E,
    ks = kt = pi E / (2 (1 + nu))), and its bonds fail in the reference's own class."""
    import math

    import pytest

    from esys.lsm import BrittleBeamDZCPrms, BrittleBeamSCPrms, LsmMpi, NRotElasticWallPrms, RotSphere
    from esys.lsm.util import BoundingBox, Vec3

    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    E, nu = 3e4, 0.25
    crit = dict(cohesion=2.0, frictionAngle=30.0, tensileCutoff=3.0, compressCutoff=10.0, beta1=1.0, beta2=1.0)
    rng = np.random.default_rng(5)
    pos = [(0.5 + (i % 3), 0.5 + (i // 3 % 3), 0.5 + (i // 9)) for i in range(18)]
    pos = [tuple(x + rng.uniform(-0.005, 0.005) for x in p) for p in pos]
    bonds = [(i, j) for i in range(18) for j in range(i + 1, 18)
             if abs(np.linalg.norm(np.subtract(pos[i], pos[j])) - 1.0) < 0.02]

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=RefBackend)
    sim.initNeighbourSearch(particleType="RotSphere", gridSpacing=1.25, verletDist=0.2)
    sim.setNumTimeSteps(150)
    sim.setTimeStepSize(1e-5)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(3, 3, 2)))
    vel = rng.normal(0, 2.0, size=(18, 3))
    parts = []
    for i, p in enumerate(pos):
        q = RotSphere(i, Vec3(*p), 0.5, float(S.sphere_mass(0.5)))
        q.setLinearVelocity(Vec3(*vel[i]))
        parts.append(q)
    sim.createParticles(parts)
    sim.createConnections([(1, i, j) for i, j in bonds])
    if law == "dzc":
        sim.createInteractionGroup(BrittleBeamDZCPrms("bb", E, nu, tag=1, **crit))
    else:
        sim.createInteractionGroup(BrittleBeamSCPrms("bb", E, nu, cohesion=20.0, frictionAngle=30.0,
                                                     tensileCutoff=20.0, tag=1))
    sim.createWall("top", Vec3(0, 3.02, 0), Vec3(0, -1, 0))
    sim.createInteractionGroup(NRotElasticWallPrms("top_w", "top", 1e5))
    sim.run()

    d = RefBackend("RotSphere", 1.25, 0.2, (0, 0, 0), (3, 3, 2), (0, 0, 0), 1e-5)
    d.add_particles(list(range(18)), [list(p) for p in pos], [0.5] * 18, [float(S.sphere_mass(0.5))] * 18,
                    tag=[0] * 18, vel=vel)
    d.add_connections([1] * len(bonds), [i for i, _ in bonds], [j for _, j in bonds])
    G = E / (2.0 * (1. + nu))
    if law == "dzc":
        d.add_brittle_beam_dzc_group("bb", 1, math.pi * E, math.pi * G, math.pi * G, math.pi * E, 2.0, 3.0, 10.0,
                                     30.0, 1.0, 1.0)
    else:
        d.add_brittle_beam_sc_group("bb", 1, math.pi * E, math.pi * G, math.pi * G, math.pi * E, 20.0, 20.0, 30.0)
    d.add_wall("top", (0, 3.02, 0), (0, -1, 0))
    d.add_wall_group("top_w", "top", 1e5)
    d.step(150)
    a, b = sim._sim.particles(), d.particles()
    for k in ("pos", "vel", "angvel"):
        assert np.array_equal(a[k], b[k]), k
    assert len(bonds) > 20 and np.abs(b["angvel"]).max() > 0
    ba, bb = sim._sim.breaks(), d.breaks()
    assert all(np.array_equal(x, y) for x, y in zip(ba, bb)) and 0 < len(bb[0]) < len(bonds)
