"""Field savers on the GPU: per-particle and per-interaction scalar fields against the
state they are computed from and against the CPU oracle, and the files the savers write.
All tests need a GPU."""
import os

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


@pytest.fixture(scope="module")
def orc(oracle_libs):
    return lambda *a: oracle_libs.OracleSim("orc", *a)


def test_kinetic_energy_fields_match_reference_formulas(gpu):
    """e_kin = (0.5 m)(v.v) + ((0.5 I) w).w for RotSpheres (Model/RotParticle.h:198-200),
    bit for bit from the particles' own state."""
    s = S.friction_pack(gpu)
    s.step(40)
    p = s.particles()
    ids, ek = s.particle_scalar_field("e_kin")
    _, el = s.particle_scalar_field("e_kin_linear")
    _, er = s.particle_scalar_field("e_kin_rot")
    _, va = s.particle_scalar_field("v_abs")
    assert np.array_equal(ids, p["id"])
    v, w = p["vel"], p["angvel"]
    vv = v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]
    assert np.array_equal(ek, el + er)
    assert np.array_equal(va, np.sqrt(vv))
    _, r = s.particle_scalar_field("radius")
    m = (4.0 / 3.0) * S.PI_REF * r * r * r
    assert np.array_equal(el, (0.5 * m) * vv)


def test_friction_fields_match_oracle_state(gpu, orc):
    a, b = S.friction_pack(gpu), S.friction_pack(orc)
    a.step(60)
    b.step(60)
    i1, i2, cnt = a.interaction_scalar_field("friction", "count")
    _, _, slip = a.interaction_scalar_field("friction", "slipping")
    _, _, stick = a.interaction_scalar_field("friction", "sticking")
    _, _, epot = a.interaction_scalar_field("friction", "potential_energy")
    o1, o2, st = b.pairs("friction")
    ref = {(int(x), int(y)): r for x, y, r in zip(o1, o2, st)}
    for k, (x, y) in enumerate(zip(i1, i2)):
        r = ref[(int(x), int(y))]
        assert cnt[k] == r[4] and slip[k] == r[3] and stick[k] == (1.0 if r[4] and not r[3] else 0.0)
    assert cnt.sum() > 0 and (epot >= 0).all() and (epot[cnt == 0] == 0).all() and epot.max() > 0


def test_bond_fields_match_oracle_criterion(gpu, orc):
    a = S.bonded_block(gpu, strength=(5.0, 5.0, 5.0, 5.0))
    b = S.bonded_block(orc, strength=(5.0, 5.0, 5.0, 5.0))
    S.run_loaded(a, 40, 0.001)
    S.run_loaded(b, 40, 0.001)
    i1, i2, crit = a.interaction_scalar_field("bonds", "breaking_criterion")
    _, _, cnt = a.interaction_scalar_field("bonds", "count")
    _, _, ep = a.interaction_scalar_field("bonds", "potential_energy")
    parts = [a.interaction_scalar_field("bonds", f)[2] for f in ("e_pot_normal", "e_pot_shear", "e_pot_twist",
                                                                 "e_pot_bend")]
    assert np.all(cnt == 1.0)
    assert np.allclose(ep, parts[0] + parts[1] + parts[2] + parts[3], rtol=1e-14, atol=0)
    o1, o2, st = b.pairs("bonds")
    ref = {(int(x), int(y)): r[3] for x, y, r in zip(o1, o2, st)}
    got = np.array([crit[k] for k in range(len(i1))])
    want = np.array([ref[(int(x), int(y))] for x, y in zip(i1, i2)])
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()


def test_lsm_field_savers_write_reference_formats(dem_lib, tmp_path):
    from esys.lsm import (InteractionScalarFieldSaverPrms, LsmMpi, NRotElasticWallPrms, ParticleScalarFieldSaverPrms,
                          RotFrictionPrms, RotSphere, WallVectorFieldSaverPrms)
    from esys.lsm.util import BoundingBox, Vec3

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1])
    sim.initNeighbourSearch("RotSphere", 1.2, 0.2)
    sim.setTimeStepSize(5e-5)
    sim.setSpatialDomain(BoundingBox(Vec3(0, -1, 0), Vec3(6, 6, 6)))
    rng = np.random.default_rng(3)
    parts = []
    for k in range(80):
        p = RotSphere(k, Vec3(*(rng.uniform(0.5, 5.5, 3))), 0.3, 0.1)
        p.setLinearVelocity(Vec3(*rng.normal(0, 0.3, 3)))
        parts.append(p)
    sim.createParticles(parts)
    sim.createInteractionGroup(RotFrictionPrms("friction", 1e4, 0.6, 0.6, 1e4))
    sim.createWall("floor", Vec3(0, 0, 0), Vec3(0, 1, 0))
    sim.createInteractionGroup(NRotElasticWallPrms("floor_w", "floor", 1e4))
    f1, f2, f3, f4 = (str(tmp_path / n) for n in ("ek.dat", "ekmax.dat", "count.dat", "wall.dat"))
    sim.createFieldSaver(ParticleScalarFieldSaverPrms("e_kin", f1, "SUM", 0, 100, 10))
    sim.createFieldSaver(ParticleScalarFieldSaverPrms("v_abs", f2, "MAX", 5, 100, 25))
    sim.createFieldSaver(InteractionScalarFieldSaverPrms("friction", "count", f3, "SUM", 0, 100, 20))
    sim.createFieldSaver(WallVectorFieldSaverPrms("floor", "Force", f4, "RAW_SERIES", 0, 100, 50))
    sim.setNumTimeSteps(100)
    sim.run()
    ek = open(f1).read().splitlines()
    assert len(ek) == 11 and all(float(x) > 0 for x in ek)
    assert len(open(f2).read().splitlines()) == 4          # steps 5, 30, 55, 80
    cnt = open(f3).read().splitlines()
    assert len(cnt) == 6 and cnt[0] == "%.10e" % 0.0      # nothing touching before the first step
    wall = open(f4).read().splitlines()
    assert len(wall) == 3 and len(wall[1].split()) == 3
    # the e_kin lines are the id-ordered sums of the particle field, printed as %g
    sim2 = sim._sim
    _, ekin = sim2.particle_scalar_field("e_kin")
    s = 0.0
    for x in ekin.tolist():
        s += x
    assert ek[-1] == "%g" % s
    sim.exit()


def _gas(make, n_side=5, with_particles=True):
    """NRotSpheres, one per x-row of a 5 x 5 (y, z) lattice, crossing the periodic x faces at
    5 to 12 per unit time: no contacts, so each one's unwrapped path is x0 + v t."""
    sim = make("NRotSphere", 1.2, 0.2, (0, 0, 0), (6, 6, 6), (1, 0, 0), 1e-3)
    sim.add_elastic_group("elastic", 1000.0, True)
    if with_particles:
        rng = np.random.default_rng(21)
        yz = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), indexing="ij"), -1).reshape(-1, 2)
        n = len(yz)
        pos = np.zeros((n, 3))
        pos[:, 0] = rng.uniform(0.5, 5.5, n)
        pos[:, 1:] = yz * 1.2 + 0.6 + rng.uniform(-0.1, 0.1, size=yz.shape)
        vel = np.zeros((n, 3))
        vel[:, 0] = rng.uniform(5.0, 12.0, n) * rng.choice([-1.0, 1.0], n)
        sim.add_particles(np.arange(n), pos, np.full(n, 0.3), np.full(n, 0.1), tag=np.zeros(n, np.int32), vel=vel)
        sim._x0, sim._v = pos, vel
    return sim


def test_vector_fields_match_particle_state(gpu):
    s = S.friction_pack(gpu)
    s.step(30)
    p = s.particles()
    for field, key in (("position", "pos"), ("velocity", "vel"), ("force", "force"), ("ang_velocity", "angvel")):
        ids, v = s.particle_vector_field(field)
        assert np.array_equal(ids, p["id"]) and np.array_equal(v, p[key]), field
    with pytest.raises(Exception):
        _gas(gpu).particle_vector_field("ang_velocity")  # NRotSpheres have no spin field


def test_displacement_follows_circular_shifts_and_checkpoints(gpu, tmp_path):
    """getTotalDisplacement = m_pos - m_initpos, with m_initpos moved by every circular shift
    (CParticle::setCircular): continuous across the periodic faces, and carried by a restart
    checkpoint's shift column (CParticle::saveCheckPointData)."""
    s = _gas(gpu)
    s.step(300)
    t = 300 * 1e-3
    ids, d = s.particle_vector_field("displacement")
    p = s.particles()
    want = s._v[ids] * t
    assert np.abs(d - want).max() < 1e-9
    wrapped = np.abs((p["pos"] - s._x0[ids])[:, 0] - d[:, 0]) > 1.0
    assert wrapped.sum() >= 5
    path = str(tmp_path / "gas_t=300_1.txt")
    s.save_checkpoint(path, 17)
    s2 = _gas(gpu, with_particles=False)
    s2.load_checkpoint(path, 300)
    _, d2 = s2.particle_vector_field("displacement")
    assert np.abs(d2 - d).max() < 1e-12
    s.step(100)
    s2.step(100)
    _, d3 = s.particle_vector_field("displacement")
    _, d4 = s2.particle_vector_field("displacement")
    assert np.abs(d3 - d4).max() < 1e-12
    assert np.abs(d3 - s._v[ids] * 0.4).max() < 1e-9


@pytest.mark.parametrize("law", ["nfric", "hm", "hmv"])
def test_nrot_friction_and_hertz_mindlin_fields(gpu, law):
    """count / slipping / sticking from the flags the step wrote, and potential_energy from the positions
    the force evaluation read: CFrictionInteraction 0.5 Fn.Fn / k + 0.5 Ff.Ff / ks (scaled k, ks), and
    CHertzMindlinInteraction and CHertzMindlinViscoInteraction 0.5 Fn.Fn / E of the elastic Hertz force."""
    sim = gpu("NRotSphere", 1.2, 0.2, (0, 0, 0), (6, 6, 6), (0, 0, 0), 1e-4)
    pos = np.array([[2.0, 2.0, 2.0], [2.85, 2.1, 2.0], [4.5, 4.5, 4.5]])
    rad = np.array([0.5, 0.45, 0.4])
    sim.add_particles(np.arange(3), pos, rad, np.ones(3), tag=np.zeros(3, np.int32),
                      vel=[[0.0, 0.3, 0.0], [0.0, -0.3, 0.1], [0.0, 0.0, 0.0]])
    if law == "nfric":
        sim.add_nrot_friction_group("c", 1e4, 0.5, 5e3, 1e-4, True)
    elif law == "hm":
        sim.add_hertz_mindlin_group("c", 1e4, 0.3, 0.5, 1e-4)
    else:
        sim.add_hertz_mindlin_visco_group("c", 1e4, 0.3, 0.5, 0.8, 1e-4)
    sim.step(1)
    pa, pb, pst = sim.pairs("c")
    by_key = {(int(x), int(y)): r for x, y, r in zip(pa, pb, pst)}
    a, b, _ = sim.interaction_scalar_field("c", "count")
    st = np.array([by_key[(int(x), int(y))] for x, y in zip(a, b)])
    fields = {f: sim.interaction_scalar_field("c", f)[2] for f in ("count", "potential_energy", "slipping", "sticking")}
    assert np.array_equal(fields["count"], st[:, 4]) and np.array_equal(fields["slipping"], st[:, 3])
    assert np.array_equal(fields["sticking"], st[:, 4] * (1 - st[:, 3]))
    q = [i for i in range(len(a)) if {int(a[i]), int(b[i])} == {0, 1}][0]
    D = pos[0] - pos[1]
    dist, eq = np.linalg.norm(D), rad[0] + rad[1]
    if law == "nfric":
        f = 0.5 * (rad[0] + rad[1])
        ke, kse = f * 1e4, f * 5e3
        Fn = D * (ke * (dist - eq) / dist)
        Ff = st[q, :3]
        want = (0.5 * Fn) @ Fn / ke + (0.5 * Ff) @ Ff / kse
    else:
        R = 1.0 / (1.0 / rad[0] + 1.0 / rad[1])
        fn = D / np.linalg.norm(D) * (4.0 / 3.0 * 1e4 * np.sqrt(R) * (eq - dist) ** 1.5)
        want = (0.5 * fn) @ fn / 1e4
    assert fields["count"][q] == 1.0
    assert abs(fields["potential_energy"][q] - want) <= 1e-12 * abs(want)
