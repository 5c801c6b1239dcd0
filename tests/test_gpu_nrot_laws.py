"""NRotFriction (CFrictionInteraction) and NRotBond (CBondedInteraction) on the GPU against the
reference's own code (the reference-built harness).  All tests need a GPU.

Bars as the core parity tests: pair sets and bond-failure events bit-exact; particle state within
1e-9 and friction histories within 1e-8 of each field's scale (summation order differs); the
checkpoint records of both laws equal the reference writer's.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


@pytest.fixture(scope="module")
def ref(oracle_libs):
    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    return lambda *a: oracle_libs.OracleSim("ref", *a)


def _by_id(p, k):
    return p[k][np.argsort(p["id"])]


def _close(x, y, rel, what):
    scale = max(np.abs(y).max(), 1e-300)
    assert np.abs(x - y).max() <= rel * scale, (what, np.abs(x - y).max() / scale)


def _pairs(sim, g):
    a, b, st = sim.pairs(g)
    return {(int(x), int(y)): s for x, y, s in zip(a, b, st)}


@pytest.mark.parametrize("rot", [False, True])
def test_nrot_friction_matches_reference(gpu, ref, rot):
    a, b = S.nrot_friction_pack(gpu, rot=rot), S.nrot_friction_pack(ref, rot=rot)
    a.step(200)
    b.step(200)
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    if rot:  # forces only: spins stay at rest
        assert np.abs(pa["angvel"]).max() == 0.0
    fa, fb = _pairs(a, "friction"), _pairs(b, "friction")
    assert fa.keys() == fb.keys()
    keys = sorted(fb)
    A = np.array([fa[k] for k in keys])
    B = np.array([fb[k] for k in keys])
    assert np.array_equal(A[:, 3:], B[:, 3:])            # slipping, touching
    assert B[:, 4].sum() > 50 and B[:, 3].sum() > 10      # contacts that stick and that slide
    _close(A[:, :3], B[:, :3], 1e-8, "history")


def test_nrot_bond_failures_match_reference(gpu, ref):
    a, b = S.nrot_bonded_block(gpu), S.nrot_bonded_block(ref)
    S.run_loaded(a, 220, a._load_rate)
    S.run_loaded(b, 220, b._load_rate)
    # a failure detected in the last step is logged for the next step's update, which the
    # reference has not run yet: compare the events up to the last step
    ea, eb = ({e for e in zip(*(x.tolist() for x in log)) if e[2] <= 220} for log in (a.breaks(), b.breaks()))
    assert len(eb) > 5
    assert ea == eb
    assert _pairs(a, "bonds").keys() == _pairs(b, "bonds").keys()
    assert _pairs(a, "friction").keys() == _pairs(b, "friction").keys()
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)


def test_nrot_checkpoint_records_match_reference(gpu, ref, tmp_path):
    """Bonded (k, r0, distance, break, scaling, ids, tag) and Friction (k, r0, mu, ks, dt, scaling,
    ids, flags, history) records of the GPU's checkpoint against the reference writer's."""
    a, b = S.nrot_bonded_block(gpu), S.nrot_bonded_block(ref)
    S.run_loaded(a, 200, a._load_rate)
    S.run_loaded(b, 200, b._load_rate)
    pa, pb = tmp_path / "g_t=200_1.txt", tmp_path / "r_t=200_1.txt"
    a.save_checkpoint(pa, 12)
    b.save_checkpoint(pb, 12)
    ca, cb = S.parse_checkpoint(pa), S.parse_checkpoint(pb)
    for sec in ("bonds", "friction"):
        assert ca[sec].keys() == cb[sec].keys() and len(cb[sec]) > 0, sec
        for k in cb[sec]:
            _close(np.array(ca[sec][k]), np.array(cb[sec][k]), 1e-8, (sec, k))


def test_nrot_restart_continues_like_the_reference(gpu, ref, tmp_path):
    """The GPU's checkpoint of an NRotBond + NRotFriction run, read by the reference and by the
    GPU; both restarted runs continue alike (failures included)."""
    a = S.nrot_bonded_block(gpu)
    S.run_loaded(a, 150, a._load_rate)
    path = tmp_path / "g_t=150_1.txt"
    a.save_checkpoint(path, 12)
    r2, g2 = S.nrot_bonded_block_script(ref), S.nrot_bonded_block_script(gpu)
    r2.load_checkpoint(path, a.timestep)
    g2.load_checkpoint(path, a.timestep)
    S.run_loaded(r2, 70, r2._load_rate)
    S.run_loaded(g2, 70, g2._load_rate)
    pa, pb = g2.particles(), r2.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    last = a.timestep + 70
    ea, eb = ({e for e in zip(*(x.tolist() for x in log)) if e[2] <= last} for log in (g2.breaks(), r2.breaks()))
    assert ea == eb and len(eb) > 0


@pytest.mark.parametrize("name", ["Alocal", "zlocal"])  # sorts before / after "Damping" in the damping map
def test_local_damping_matches_reference(gpu, ref, name):
    """LocalDamping (with the viscous linear damping, ordered by group name) on an NRotSphere
    gravity packing, and LocalDamping + RotLocalDamping with both viscous dampings on a
    rotational friction pack."""
    a, b = S.gravity_box(gpu, n_side=5), S.gravity_box(ref, n_side=5)
    for s in (a, b):
        s.add_local_damping(name, 0, 0.3)
        s.step(200)
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    a, b = S.loaded_friction_pack(gpu), S.loaded_friction_pack(ref)
    for s in (a, b):
        s.add_local_damping(name, 0, 0.2)
        s.add_local_damping("rotlocal", 1, 0.2)
        s.step(150)
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "angvel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)


@pytest.mark.parametrize("rot", [False, True])
def test_hertz_mindlin_matches_reference(gpu, ref, rot):
    """HertzMindlin (CHertzMindlinInteraction) through several neighbour rebuilds, which restart
    its tangential history (PIS_NE storage) in the reference and here alike."""
    a, b = S.hertz_mindlin_pack(gpu, rot=rot), S.hertz_mindlin_pack(ref, rot=rot)
    c0 = a.counters()["rebuilds"]
    a.step(300)
    b.step(300)
    assert a.counters()["rebuilds"] - c0 >= 2
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    fa, fb = _pairs(a, "hm"), _pairs(b, "hm")
    assert fa.keys() == fb.keys()
    keys = sorted(fb)
    A = np.array([fa[k] for k in keys])
    B = np.array([fb[k] for k in keys])
    assert np.array_equal(A[:, 3:], B[:, 3:])
    assert B[:, 4].sum() > 50 and B[:, 3].sum() > 10
    _close(A[:, :3], B[:, :3], 1e-8, "history")


def test_brittle_beam_dzc_failures_match_reference(gpu, ref):
    """BrittleBeamDZC (BrittleBeamDZCInteraction): RotBond forces and moments, the beam-stress
    failure criterion; failure events exact, state within 1e-9 of the reference's own class."""
    a, b = S.dzc_block(gpu), S.dzc_block(ref)
    S.run_loaded(a, 400, 2e-4)
    S.run_loaded(b, 400, 2e-4)
    ea, eb = ({e for e in zip(*(x.tolist() for x in log)) if e[2] <= 400} for log in (a.breaks(), b.breaks()))
    assert len(eb) > 20 and len({e[2] for e in eb}) > 10  # failures spread over the run
    assert ea == eb
    assert _pairs(a, "bonds").keys() == _pairs(b, "bonds").keys()
    assert _pairs(a, "friction").keys() == _pairs(b, "friction").keys()
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "angvel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    with pytest.raises(Exception):
        a.save_checkpoint("unused_t=1_1.txt", 12)  # restart records of these groups are not built


def test_brittle_beam_sc_failures_match_reference(gpu, ref):
    """BrittleBeamSC (BrittleBeamSCInteraction): RotBond forces; failure at the update from the
    particles' stress sums (CParticle::applyForce's m_sigma) of the step before.  Failure events
    exact, state within 1e-9 of the reference's own class."""
    a, b = S.sc_block(gpu), S.sc_block(ref)
    S.run_loaded(a, 400, 2e-4)
    S.run_loaded(b, 400, 2e-4)
    ea, eb = ({e for e in zip(*(x.tolist() for x in log))} for log in (a.breaks(), b.breaks()))
    assert len(eb) > 10 and len({e[2] for e in eb}) > 8
    assert ea == eb
    assert _pairs(a, "bonds").keys() == _pairs(b, "bonds").keys()
    assert _pairs(a, "friction").keys() == _pairs(b, "friction").keys()
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "angvel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)


@pytest.mark.parametrize("rot,restitution", [(False, 0.6), (True, 0.6), (True, 0.95)])
def test_hertz_mindlin_visco_matches_reference(gpu, ref, rot, restitution):
    """HertzMindlinVisco (CHertzMindlinViscoInteraction): damped Hertz-Mindlin contacts through several
    neighbour rebuilds, state within 1e-9 of the reference's own class, and the slipping / sticking
    interaction fields equal to its getSlipping / getSticking; restitution 0.95 leaves little damping."""
    a = S.hertz_mindlin_pack(gpu, rot=rot, restitution=restitution)
    b = S.hertz_mindlin_pack(ref, rot=rot, restitution=restitution)
    c0 = a.counters()["rebuilds"]
    a.step(300)
    b.step(300)
    assert a.counters()["rebuilds"] - c0 >= 2
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    c = a.interaction_scalar_field("hm", "count")[2]
    assert c.sum() > 20
    ia, ib, _ = a.interaction_scalar_field("hm", "slipping")
    fa = {f: dict(zip(zip(ia.tolist(), ib.tolist()), a.interaction_scalar_field("hm", f)[2]))
          for f in ("slipping", "sticking")}
    ra, rb, rst = b.pairs("hm")
    rb_map = {(int(x), int(y)): r for x, y, r in zip(ra, rb, rst)}
    common = [k for k in fa["slipping"] if k in rb_map]
    assert len(common) > 20
    for k in common:
        assert fa["slipping"][k] == rb_map[k][3], k
        assert fa["sticking"][k] == rb_map[k][4] - rb_map[k][3], k
