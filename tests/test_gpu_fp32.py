"""The FP32-force / FP64-integration form (precision form 1).

Bar: forces of the FP32 form evaluated on the same state as the FP64 form are
within 1e-5 of the largest force magnitude (the spec's relative force error),
the contact (pair) set is identical, and short FP32 trajectories stay within
1e-6 of the FP64 ones."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _check(sim):
    import ctypes

    out = (ctypes.c_double * 5)()
    rc = sim.lib.dem_precision_check(sim.h, out)
    assert rc == 0, sim.lib.dem_last_error(sim.h)
    return list(out)


@pytest.mark.parametrize("tpp", [1, 2, 4, 16, 32])
def test_fp32_force_error_friction(gpu, tpp):
    s = S.friction_pack(gpu)
    s.set_option("threads_per_particle", tpp)
    s.step(150)
    err = _check(s)
    assert err[4] > 50
    assert err[0] <= 1e-5, err
    assert err[1] <= 1e-5, err


def test_fp32_force_error_elastic_nrot(gpu):
    s = S.gravity_box(gpu, 6)
    s.step(150)
    err = _check(s)
    assert err[0] <= 1e-5, err


@pytest.mark.parametrize("split", [0, 1])
def test_fp32_trajectory_close_to_fp64(gpu, split):
    a, b = S.friction_pack(gpu), S.friction_pack(gpu)
    b.set_option("precision", 32)
    b.set_option("split", split)
    a.step(100)
    b.step(100)
    pa, pb = a.particles(), b.particles()
    assert np.abs(pa["pos"] - pb["pos"]).max() <= 1e-6 * np.abs(pa["pos"]).max()
    x, y = a.pairs("friction"), b.pairs("friction")
    assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    # history is stored in FP32 in the FP32 form
    assert np.abs(x[2][:, :3] - y[2][:, :3]).max() <= 1e-4 * max(np.abs(x[2][:, :3]).max(), 1e-30)


def test_fp32_switch_midway_keeps_history(gpu):
    a, b = S.friction_pack(gpu), S.friction_pack(gpu)
    a.step(80)
    b.step(80)
    b.set_option("precision", 32)
    b.step(20)
    b.set_option("precision", 64)
    b.step(20)
    a.step(40)
    pa, pb = a.particles(), b.particles()
    assert np.abs(pa["vel"] - pb["vel"]).max() <= 1e-4 * np.abs(pa["vel"]).max()


def test_fp32_bonded_block_force_error(gpu):
    """Bonded, loaded, breaking block: the FP32 form takes its bond forces from the FP64
    (uncontracted) bond pass, so only the RotFriction contacts carry FP32 rounding; the error
    stays far under 1e-5 both against the largest force and per particle against its own
    contact-force scale."""
    s = S.bonded_block(gpu, strength=(0.3, 0.6, 0.6, 0.3))
    s.set_option("precision", 32)
    S.run_loaded(s, 120, 0.002)
    assert len(s.breaks()[0]) > 0
    s.set_option("precision", 64)
    r = s.precision_report()
    assert r["max_rel_force_err"] <= 1e-6, r
    assert r["rel_to_force_scale"] <= 1e-6, r
    assert r["worst_rel_to_own_scale"] <= 1e-5, r
