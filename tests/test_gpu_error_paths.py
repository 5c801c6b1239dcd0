"""Error paths of the library on the GPU.  All tests need a GPU.

Every failure is made on the host or by a capacity the test sets: unknown wall and
group names, bad options and counts come back as DEM_ERR_ARG with the reference's
message where it has one (SubLattice.hpp:688-692 "not found in map of walls",
1980-2009 "nonexisting interaction group"); a bond-break event log made too small
fills and the call in which it filled returns DEM_ERR_OVERFLOW, with the bond states
exact; the damping fixed point capped at maxIterations (Damping.hpp:116-119) matches
the CPU restatement.  After each failure the handle goes on stepping and matches a
twin that never saw the bad call.
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
def orc(oracle_libs):
    return lambda *a: oracle_libs.OracleSim("orc", *a)


def _same(a, b, groups):
    pa, pb = a.particles(), b.particles()
    for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(pa[k], pb[k]), k
    for g in groups:
        x, y = a.pairs(g), b.pairs(g)
        for u, v in zip(x, y):
            assert np.array_equal(u, v), g


def _arg_error(fn, *frags):
    from esys.lsm import _capi

    with pytest.raises(_capi.DemError) as e:
        fn()
    assert e.value.status == _capi.DEM_ERR_ARG, (e.value.status, str(e.value))
    for f in frags:
        assert f in str(e.value), (f, str(e.value))


def test_unknown_names_and_bad_arguments_leave_the_handle_usable(gpu):
    a = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    b = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    a.step(5)
    b.step(5)
    _arg_error(lambda: a.move_wall("no_such_wall", (0, 1, 0)), "no such wall")
    _arg_error(lambda: a.set_wall_velocity("no_such_wall", (0, 1, 0)), "no such wall")
    _arg_error(lambda: a.wall("no_such_wall"), "no such wall")
    _arg_error(lambda: a.add_wall_group("w2", "no_such_wall", 1e5), "not found in map of walls")
    _arg_error(lambda: a.apply_force_to_wall("no_such_group", (0, 1, 0)))
    _arg_error(lambda: a.add_exclusion("no_such_group", "friction"), "nonexisting interaction group")
    _arg_error(lambda: a.add_exclusion("bonds", "no_such_group"), "nonexisting interaction group")
    _arg_error(lambda: a.pairs("no_such_group"))
    _arg_error(lambda: a.interaction_scalar_field("no_such_group", "potential_energy"))
    _arg_error(lambda: a.set_group_param("no_such_group", "normalK", 1.0))
    _arg_error(lambda: a.set_option("no_such_option", 1), "unknown option")
    _arg_error(lambda: a.set_option("threads_per_particle", 3), "threads_per_particle")
    _arg_error(lambda: a.set_option("event_capacity", -1), "event_capacity")
    _arg_error(lambda: a.set_option("event_capacity", 2.5), "event_capacity")
    _arg_error(lambda: a.step(-1), "negative step count")
    _arg_error(lambda: a.set_timestep(0.0), "time step")
    _arg_error(lambda: a.add_particles([0], [[1.0, 1.0, 1.0]], [0.4], [1.0]), "duplicate particle id")
    _arg_error(lambda: a.add_particles([999], [[1.0, 1.0, 1.0]], [0.0], [1.0]), "radius and mass")
    S.run_loaded(a, 100, 2e-4)
    S.run_loaded(b, 100, 2e-4)
    _same(a, b, ["bonds", "friction"])
    for w in ("top", "bottom"):
        assert np.array_equal(a.wall(w)[1], b.wall(w)[1]), w


def test_rot_damping_needs_rotational_particles(gpu):
    sim = S.gravity_box(gpu, 3)
    _arg_error(lambda: sim.add_damping(1, 0.01, 50), "RotDamping needs RotSphere")
    _arg_error(lambda: sim.add_local_damping("", 0, 0.01), "name of its own")


def test_periodic_x_range_is_adjusted_like_the_reference(gpu, orc):
    """A periodic x side that is no multiple of the range: the range becomes side /
    floor(side / range) (SubLattice.hpp:506-515), here 10 / 3 from 3.0, with
    particles on both sides of the seam; the pair set and state match the oracle."""
    rng = np.random.default_rng(11)
    g = np.stack(np.meshgrid(np.arange(10), np.arange(3), np.arange(3), indexing="ij"), -1).reshape(-1, 3)
    n = len(g)
    # x centres 0.5 .. 9.5: the first and last columns touch across the seam
    pos = g + np.array([0.5, 1.0, 1.0]) + rng.uniform(-0.02, 0.02, g.shape)
    rad = rng.uniform(0.48, 0.52, n)
    vel = rng.normal(0, 0.1, (n, 3))
    sims = []
    for make in (gpu, orc):
        s = make("RotSphere", 3.0, 0.2, (0, 0, 0), (10, 4, 4), (1, 0, 0), 1e-4)
        s.add_particles(np.arange(n), pos, rad, S.sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel)
        s.add_rot_friction_group("friction", 1e4, 0.6, 0.6, 1e4, 1e-4, True, True)
        s.step(200)
        sims.append(s)
    a, b = sims
    pa, pb = a.particles(), b.particles()
    assert np.array_equal(pa["id"], pb["id"])
    for k in ("pos", "vel", "angvel", "force", "moment"):
        assert np.abs(pa[k] - pb[k]).max() <= 1e-8 * max(np.abs(pb[k]).max(), 1e-300), k
    x, y = a.pairs("friction"), b.pairs("friction")
    assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    seam = {(i, j) for i, j in zip(x[0].tolist(), x[1].tolist()) if abs(pa["pos"][i, 0] - pa["pos"][j, 0]) > 5}
    assert seam, "pairs across the periodic seam"


def _loaded_with_log(sim, steps, rate):
    """run_loaded that records the calls returning DEM_ERR_OVERFLOW instead of stopping."""
    from esys.lsm import _capi

    overflow_calls = []
    for i in range(steps):
        sim.move_wall("top", (0, -rate, 0))
        sim.move_wall("bottom", (0, rate, 0))
        try:
            sim.step(1)
        except _capi.DemError as e:
            assert e.status == _capi.DEM_ERR_OVERFLOW, str(e)
            assert "bond states are exact" in str(e)
            overflow_calls.append(i)
    return overflow_calls


@pytest.mark.parametrize("cap", [1, 3])
def test_event_log_overflow_reports_and_keeps_bond_states_exact(gpu, cap):
    full = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    small = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    small.set_option("event_capacity", cap)
    assert _loaded_with_log(full, 400, 2e-4) == []
    calls = _loaded_with_log(small, 400, 2e-4)
    ef, es = full.breaks(), small.breaks()
    nfull = len(ef[0])
    assert nfull > cap, "the case must break more bonds than the log holds"
    assert len(calls) >= 1 and small.timestep == full.timestep
    # the logged events are the first `cap` failures (by step) of the full log
    assert len(es[0]) == cap
    logged = set(zip(*[x.tolist() for x in es]))
    assert logged <= set(zip(*[x.tolist() for x in ef]))
    first_steps = sorted(ef[2].tolist())[:cap]
    assert sorted(es[2].tolist()) == first_steps
    # the simulation itself is the full-log one, bit for bit
    _same(small, full, ["bonds", "friction"])
    # a log that has overflowed keeps its capacity
    _arg_error(lambda: small.set_option("event_capacity", 0), "has overflowed")


def test_event_capacity_cannot_drop_below_logged_events(gpu):
    sim = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    S.run_loaded(sim, 400, 2e-4)
    n = len(sim.breaks()[0])
    assert n >= 2
    _arg_error(lambda: sim.set_option("event_capacity", n - 1), "below the events already logged")
    sim.set_option("event_capacity", n + 5)
    sim.set_option("event_capacity", 0)
    assert len(sim.breaks()[0]) == n


@pytest.mark.parametrize("max_iter", [0, 1, 3, 5, 100])
@pytest.mark.parametrize("precision", [64, 32])
def test_damping_iteration_cap_matches_the_oracle(gpu, orc, max_iter, precision):
    """CDamping / CRotDamping with maxIterations 0 and 1 (never damped), 3 and 5 (fast
    particles capped, slow ones damped) and 100 (all damped); the damping runs on the
    FP64 accumulated force in both forms, so the FP32 form is held to its force bar."""
    a, b = S.damped_cloud(gpu, max_iter=max_iter), S.damped_cloud(orc, max_iter=max_iter)
    if precision == 32:
        a.set_option("precision", 32)
    a.step(20)
    b.step(20)
    pa, pb = a.particles(), b.particles()
    assert np.array_equal(pa["id"], pb["id"])
    tol = 1e-12 if precision == 64 else 1e-6
    for k in ("pos", "vel", "angvel", "force", "moment"):
        assert np.abs(pa[k] - pb[k]).max() <= tol * max(np.abs(pb[k]).max(), 1e-300), k
