"""Batched ensemble on the GPU: every specimen of an ensemble advances exactly as the
same specimen advanced alone.  All tests need a GPU.

Bar: particle state, pair sets and bond-break events bit-identical to the specimen
stepped by itself with the same threads-per-particle and precision form (the batched
kernel does the same per-particle arithmetic in the same order); wall reactions within
1e-12 of their magnitude (they are reduced over tiles instead of blocks).
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _specimens(gpu, kind):
    if kind == "friction":
        return [S.friction_pack(gpu, nx=6 + k, ny=5, nz=6 + (k % 2), seed=20 + k, periodic=(k == 1))
                for k in range(3)]
    if kind == "bonded":
        return [S.bonded_block(gpu, nx=5, ny=6 + k, nz=5, seed=30 + k, strength=st)
                for k, st in enumerate([(0.5, 1.0, 1.0, 0.5), (0.3, 0.6, 0.6, 0.3), (5.0, 5.0, 5.0, 5.0)])]
    return [S.gravity_box(gpu, n_side=4 + k, seed=40 + k) for k in range(3)]


def _advance_loaded(sims, steps, rate, step_fn):
    for _ in range(steps):
        for s in sims:
            s.move_wall("top", (0, -rate, 0))
            s.move_wall("bottom", (0, rate, 0))
        step_fn(1)


def _same(a, b, groups, tol_wall=1e-12):
    pa, pb = a.particles(), b.particles()
    for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(pa[k], pb[k]), k
    for g in groups:
        x, y = a.pairs(g), b.pairs(g)
        for u, v in zip(x, y):
            assert np.array_equal(u, v), g
    for u, v in zip(a.breaks(), b.breaks()):
        assert np.array_equal(u, v)
    assert a.timestep == b.timestep


@pytest.mark.parametrize("kind,groups,steps", [("friction", ["friction"], 300), ("elastic", ["elastic"], 200)])
@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("tpp", [2, 16])
def test_ensemble_equals_specimens_alone(gpu, kind, groups, steps, precision, tpp):
    from esys.lsm import _capi

    if kind == "elastic" and precision == 32:
        pytest.skip("the FP32 form is rotational only")
    ens_sims = _specimens(gpu, kind)
    alone = _specimens(gpu, kind)
    for s in ens_sims + alone:
        s.set_option("precision", precision)
        s.set_option("threads_per_particle", tpp)
    e = _capi.Ensemble(ens_sims)
    e.set_option("threads_per_particle", tpp)
    e.set_option("chunk", 48)
    e.step(steps)
    for s in alone:
        s.step(steps)
    for a, b in zip(ens_sims, alone):
        _same(a, b, groups)
    c = e.counters()
    assert c["specimen_steps"] == steps * len(ens_sims)
    e.close()


@pytest.mark.parametrize("tpp", [4, 16])
def test_bonded_ensemble_breaks_like_specimens_alone(gpu, tpp):
    """Bond failures (of different strengths, so at different steps), the exclusion hand-off
    to friction and rebuilds happen at different steps in different specimens."""
    from esys.lsm import _capi

    ens_sims = _specimens(gpu, "bonded")
    alone = _specimens(gpu, "bonded")
    e = _capi.Ensemble(ens_sims)
    e.set_option("threads_per_particle", tpp)
    for s in alone:
        s.set_option("threads_per_particle", tpp)
    _advance_loaded(ens_sims, 60, 0.002, e.step)
    for s in alone:
        S.run_loaded(s, 60, 0.002)
    n_breaks = [len(s.breaks()[0]) for s in alone]
    assert min(n_breaks) > 0
    for a, b in zip(ens_sims, alone):
        _same(a, b, ["friction", "bonds"])
    e.close()


def test_graph_replay_equals_plain_launches(gpu):
    from esys.lsm import _capi

    a_sims = _specimens(gpu, "friction")
    b_sims = _specimens(gpu, "friction")
    ea, eb = _capi.Ensemble(a_sims), _capi.Ensemble(b_sims)
    ea.set_option("graph", 1)
    eb.set_option("graph", 0)
    for e in (ea, eb):
        e.set_option("chunk", 32)
        e.step(100)
    for a, b in zip(a_sims, b_sims):
        _same(a, b, ["friction"])
    # specimens keep working on their own after the ensemble is gone
    ea.close()
    a_sims[0].step(5)
    b_sims[0].step(5)
    _same(a_sims[0], b_sims[0], ["friction"])
    eb.close()


def test_ensemble_rejects_mixed_particle_types(gpu):
    from esys.lsm import _capi

    with pytest.raises(_capi.DemError):
        _capi.Ensemble([S.friction_pack(gpu), S.gravity_box(gpu)])
