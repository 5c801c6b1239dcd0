"""Device bond hand-off (dem_set_option "bond_handoff"): bond failures need no host update.

The RotFriction list keeps the pairs that an intact bond excludes, skips them while the
bond holds and treats them as ordinary pairs from the step after it fails; wall candidacy
is refreshed on the device at that step.  The reference instead appends a "new list" of
both-flagged pairs at that step (ntable.hpp:628-664, pi_storage_ed.hpp:130-155).  Bar:
particle state, forces and bond-break events bit-identical to the host hand-off; the
reported friction pairs are the host list's touching pairs, the host list only adding
new-list pairs that never touched.  All tests need a GPU.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _pairs(sim):
    a, b, st = sim.pairs("friction")
    return {(int(x), int(y)): tuple(r) for x, y, r in zip(a, b, st)}


@pytest.mark.parametrize("precision", [64, 32])
def test_handoff_equals_host_handoff(gpu, precision):
    host = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3))
    dev = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3))
    for s in (host, dev):
        s.set_option("precision", precision)
    dev.set_option("bond_handoff", 1)
    S.run_loaded(host, 150, 0.002)
    S.run_loaded(dev, 150, 0.002)
    ph, pd = host.particles(), dev.particles()
    for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(ph[k], pd[k]), k
    bh, bd = host.breaks(), dev.breaks()
    assert len(bh[0]) > 0
    for u, v in zip(bh, bd):
        assert np.array_equal(u, v)
    hp, dp = _pairs(host), _pairs(dev)
    assert set(dp) <= set(hp)
    for k in dp:
        assert hp[k] == dp[k], k
    for k in set(hp) - set(dp):  # new-list pairs that never came into contact
        assert hp[k][4] == 0.0 and hp[k][0] == hp[k][1] == hp[k][2] == 0.0, k
    assert np.array_equal(host.wall("top")[1], dev.wall("top")[1])


@pytest.mark.parametrize("precision,tpp", [(64, 1), (32, 1), (64, 16), (32, 16), (64, 32), (32, 32)])
def test_handoff_equals_host_handoff_in_each_step_form(gpu, precision, tpp):
    """Lane, tiled (16) and warp-cooperative (32) step forms with the bond pass.  A held pair is
    recognised from a bit of its adjacency entry; only a particle that a failure has flagged reads
    its bond's failure step, so the block has both kinds, and pairs of broken bonds that touch."""
    host = S.bonded_block(gpu, nx=6, ny=8, nz=6, strength=(0.3, 0.6, 0.6, 0.3))
    dev = S.bonded_block(gpu, nx=6, ny=8, nz=6, strength=(0.3, 0.6, 0.6, 0.3))
    for s in (host, dev):
        s.set_option("precision", precision)
        s.set_option("bond_pass", 1)
        s.set_option("threads_per_particle", tpp)
    dev.set_option("bond_handoff", 1)
    S.run_loaded(host, 200, 0.002)
    S.run_loaded(dev, 200, 0.002)
    ph, pd = host.particles(), dev.particles()
    for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(ph[k], pd[k]), k
    bh, bd = host.breaks(), dev.breaks()
    for u, v in zip(bh, bd):
        assert np.array_equal(u, v)
    flagged = np.unique(np.concatenate([bh[0], bh[1]]))
    assert 0 < len(flagged) < len(ph["id"])
    hp, dp = _pairs(host), _pairs(dev)
    broken = {(int(min(a, b)), int(max(a, b))) for a, b in zip(bh[0], bh[1])}
    assert any(dp[k][4] != 0.0 for k in broken if k in dp)  # pairs of broken bonds in contact
    for k in dp:
        assert hp[k] == dp[k], k


@pytest.mark.parametrize("tpp", [1, 32])
def test_exclusion_added_while_running_under_handoff(gpu, tpp):
    """TSubLattice::setExIG on lists that already hold bonded pairs (SubLattice.hpp:1980-2009): the
    host path removes them, the hand-off keeps and marks them held; the runs stay bit-identical.
    The lanes are fixed: with several lanes per particle the entries a lane sums depend on the
    list's length, which differs between the two paths (held pairs stay in the hand-off's list)."""
    host = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3), with_friction=False)
    dev = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3), with_friction=False)
    for s in (host, dev):
        s.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, 1e-5, True, True)
        s.set_option("bond_pass", 1)
        s.set_option("threads_per_particle", tpp)
    dev.set_option("bond_handoff", 1)
    for s in (host, dev):
        S.run_loaded(s, 5, 0.002)
        s.add_exclusion("bonds", "friction")
        S.run_loaded(s, 150, 0.002)
    ph, pd = host.particles(), dev.particles()
    for k in ("pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(ph[k], pd[k]), k
    bh, bd = host.breaks(), dev.breaks()
    assert len(bh[0]) > 0
    for u, v in zip(bh, bd):
        assert np.array_equal(u, v)


def test_handoff_does_not_stop_chunks(gpu):
    host = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3))
    dev = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3))
    dev.set_option("bond_handoff", 1)
    for s in (host, dev):
        s.set_wall_velocity("top", (0, -200.0, 0))
        s.set_wall_velocity("bottom", (0, 200.0, 0))
        s.step(120)
    assert np.array_equal(host.particles()["pos"], dev.particles()["pos"])
    assert len(host.breaks()[0]) > 0
    assert dev.counters()["launches"] < host.counters()["launches"]


def test_handoff_ensemble_equals_specimens_alone(gpu):
    from esys.lsm import _capi

    def specs():
        out = [S.bonded_block(gpu, nx=5, ny=6 + k, nz=5, seed=50 + k, strength=(0.2 + 0.2 * k, 0.5, 0.5, 0.3))
               for k in range(3)]
        for s in out:
            s.set_option("bond_handoff", 1)
            s.set_option("threads_per_particle", 4)
            s.set_wall_velocity("top", (0, -100.0, 0))
            s.set_wall_velocity("bottom", (0, 100.0, 0))
        return out

    a, b = specs(), specs()
    e = _capi.Ensemble(a)
    e.set_option("threads_per_particle", 4)
    e.step(150)
    for s in b:
        s.step(150)
    for x, y in zip(a, b):
        px, py = x.particles(), y.particles()
        for k in ("pos", "vel", "angvel", "quat", "force", "moment"):
            assert np.array_equal(px[k], py[k]), k
        for u, v in zip(x.breaks(), y.breaks()):
            assert np.array_equal(u, v)
    e.close()


def test_handoff_needs_friction_only_groups(gpu):
    from esys.lsm._capi import DemError

    g = S.gravity_box(gpu, n_side=4)
    with pytest.raises(DemError, match="RotFriction"):
        g.set_option("bond_handoff", 1)
