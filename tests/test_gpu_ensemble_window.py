"""Batched differentiable windows (dem_ensemble_window_forward / _adjoint): every specimen's
window and reverse pass, run together with one launch per kernel and timestep, equal the
same specimen's own window.  All tests need a GPU.

Bars: reactions within 1e-12 of their magnitude (the batched step reduces wall reactions
over tiles instead of blocks); bond failures identical; gradients bit-identical (the same
recompute per particle and the same reverse arithmetic, reduced in the same fixed order).
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

T, K = 120, 32


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _specimens(gpu, precision, handoff=True, strengths=(2000.0, 1e6, 2500.0)):
    sims = [S.window_block(gpu, nx=4 + k % 2, ny=5 + k, nz=4, seed=50 + k, friction=True, strength=st)
            for k, st in enumerate(strengths)]
    for s in sims:
        if handoff:
            s.set_option("bond_handoff", 1)
        s.set_option("precision", precision)
        s.set_option("threads_per_particle", 2)
    return sims


@pytest.mark.parametrize("precision", [64, 32])
def test_ensemble_window_equals_specimens_alone(gpu, precision):
    from esys.lsm import _capi

    ens, alone = _specimens(gpu, precision), _specimens(gpu, precision)
    for k, (a, b) in enumerate(zip(ens, alone)):  # the specimens start their windows at different steps
        a.step(3 * k)
        b.step(3 * k)
    e = _capi.Ensemble(ens)
    e.set_option("threads_per_particle", 2)
    Re = e.window_forward(T, K)
    Ra = [b.window_forward(T, K) for b in alone]
    for x, y in zip(Re, Ra):
        assert np.abs(x - y).max() <= 1e-12 * np.abs(y).max()
    assert len(alone[0].breaks()[0]) > 0
    for a, b in zip(ens, alone):
        for u, v in zip(a.breaks(), b.breaks()):
            assert np.array_equal(u, v)
    gR = [S.mse_grad(y, S.mse_target(y)) for y in Ra]
    ge = e.window_adjoint(gR)
    ga = [b.window_adjoint(g) for b, g in zip(alone, gR)]
    for x, y in zip(ge, ga):
        for k in ("params", "vel", "angvel", "id"):
            assert np.array_equal(x[k], y[k]), k
        assert np.abs(x["params"]).max() > 0
    # the specimens carry on (and can be rewound) as after their own windows
    e.step(5)
    for b in alone:
        b.step(5)
    for a, b in zip(ens, alone):
        pa, pb = a.particles(), b.particles()
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(pa[k], pb[k]), k
    e.close()


def test_ensemble_window_names_the_failing_specimen(gpu):
    from esys.lsm import _capi
    from esys.lsm._capi import DemError

    # without the device hand-off a bond failure may not fall inside a window
    ens = _specimens(gpu, 64, handoff=False, strengths=(1e6, 2000.0))
    e = _capi.Ensemble(ens)
    with pytest.raises(DemError, match="specimen 1: a bond broke"):
        e.window_forward(T, K)
    e.close()


def test_search_neighbors_is_force_neutral(gpu):
    """An extra neighbour search (dem_search_neighbors) changes no force: only non-touching
    pairs leave or join the lists.  Per-particle sums may regroup (lanes take other pairs),
    so the bar is the last bits, 1e-12 of each field's scale after 60 steps."""
    a, b = _specimens(gpu, 64, strengths=(2000.0,))[0], _specimens(gpu, 64, strengths=(2000.0,))[0]
    a.step(20)
    b.step(20)
    c0 = b.counters()["rebuilds"] - a.counters()["rebuilds"]
    b.search_neighbors()
    a.step(60)
    b.step(60)
    assert b.counters()["rebuilds"] - a.counters()["rebuilds"] == c0 + 1
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "angvel"):
        scale = np.abs(pa[k]).max()
        assert np.abs(pa[k] - pb[k]).max() <= 1e-12 * scale, k
    for u, v in zip(a.breaks(), b.breaks()):
        assert np.array_equal(u, v)
