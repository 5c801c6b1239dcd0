"""The warp-cooperative pair sums (threads_per_particle = 32): a warp's adjacency entries taken
32 at a time, each touching entry's contributions sent to its particle's lane in entry order.
Each particle adds the same contributions in the same order as the one-lane loop (TPP = 1), so
in the FP64 form (built without FMA contraction) the runs are bit-identical; the instances it
does not cover (widened laws, in-line bonds, stress sums) run the one-lane loop.  All tests
need a GPU."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _state(sim, groups):
    p = sim.particles()
    out = [p[k] for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment")]
    for g in groups:
        out += list(sim.pairs(g))
    return out


def _identical(a, b, groups):
    for x, y in zip(_state(a, groups), _state(b, groups)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("periodic", [False, True])
def test_friction_pack_fp64_bit_identical_to_one_lane(gpu, periodic):
    a, b = S.friction_pack(gpu, periodic=periodic), S.friction_pack(gpu, periodic=periodic)
    a.set_option("threads_per_particle", 1)
    b.set_option("threads_per_particle", 32)
    a.step(300)
    b.step(300)
    _identical(a, b, ["friction"])
    for w in ("floor", "roof"):
        assert np.array_equal(a.wall(w)[1], b.wall(w)[1])


def test_gravity_box_fp64_bit_identical_to_one_lane(gpu):
    a, b = S.gravity_box(gpu, 6), S.gravity_box(gpu, 6)
    a.set_option("threads_per_particle", 1)
    b.set_option("threads_per_particle", 32)
    a.step(300)
    b.step(300)
    _identical(a, b, ["elastic"])


def test_bonded_block_with_bond_pass_bit_identical_to_one_lane(gpu):
    """Friction with the device bond hand-off (held pairs skipped) and gathered bond records."""
    a = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    b = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    for s, t in ((a, 1), (b, 32)):
        s.set_option("bond_pass", 1)
        s.set_option("bond_handoff", 1)
        s.set_option("threads_per_particle", t)
        S.run_loaded(s, 300, 2e-4)
    _identical(a, b, ["friction", "bonds"])
    for x, y in zip(a.breaks(), b.breaks()):
        assert np.array_equal(x, y)
    assert len(a.breaks()[0]) > 0


def test_fp32_form_close_to_one_lane(gpu):
    a, b = S.friction_pack(gpu), S.friction_pack(gpu)
    for s, t in ((a, 1), (b, 32)):
        s.set_option("precision", 32)
        s.set_option("threads_per_particle", t)
        s.step(200)
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "force", "moment"):
        assert np.abs(pa[k] - pb[k]).max() <= 1e-6 * max(np.abs(pb[k]).max(), 1e-300), k
    x, y = a.pairs("friction"), b.pairs("friction")
    assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


def test_uncovered_instances_fall_back_to_one_lane(gpu):
    """NRotFriction (a widened law) with threads_per_particle = 32 runs the one-lane loop."""
    a, b = S.nrot_friction_pack(gpu), S.nrot_friction_pack(gpu)
    a.set_option("threads_per_particle", 1)
    b.set_option("threads_per_particle", 32)
    a.step(100)
    b.step(100)
    _identical(a, b, [])
