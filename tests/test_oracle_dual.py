"""The dual-number window of the CPU restatement: the checker of the GPU adjoint.

Pinned on the CPU two ways.  Its values equal the restatement's own FP64 steps
bit for bit (same laws, same operation order).  Its derivatives of a
platen-force MSE agree with FP64 central finite differences of the
restatement to 1e-4 relative.  The finite differences are taken at
h = 1e-6 ... 1e-2 relative (decades) and the best of them must agree: the
200-step loss carries FP64 rounding noise of ~1e-10 relative (a bouncing,
loaded block amplifies the last-bit differences of two runs), so a 1e-6 step
resolves only the strongest inputs, while the larger steps' truncation error
stays below 1e-6 for this smooth window.  Every step's error is in the
assertion message.
"""
import numpy as np
import pytest

import scenarios as S

T = 200


@pytest.fixture(scope="module")
def orc(oracle_libs):
    return lambda *a: oracle_libs.OracleSim("orc", *a)


def test_dual_values_equal_fp64_steps(orc):
    a = S.window_block(orc)
    a.step(10)
    R, dR = a.window_dual(60, list(S.WINDOW_SEEDS), 2)
    ref = S.wall_force_history(a, 60)
    assert np.array_equal(R, ref)
    assert np.abs(R).max() > 0 and np.abs(dR).max() > 0


def central_difference(loss_at, base, rel):
    h = rel * max(abs(base), 1e-3)
    return (loss_at(base + h) - loss_at(base - h)) / (2 * h)


def check_gradient(g, loss_at, base, rtol=1e-4):
    errs = {}
    for rel in (1e-6, 1e-5, 1e-4, 1e-3, 1e-2):
        g_fd = central_difference(loss_at, base, rel)
        errs[rel] = abs(g - g_fd) / abs(g_fd)
    assert min(errs.values()) <= rtol, (g, errs)


@pytest.fixture(scope="module")
def dual_run(orc):
    a = S.window_block(orc)
    p = a.particles()
    i1, i2, _ = a.pairs("bonds")
    bonded = np.isin(p["id"], np.concatenate([i1, i2]))
    y = np.where(bonded, p["pos"][:, 1], np.nan)
    lo, hi = int(p["id"][np.nanargmin(y)]), int(p["id"][np.nanargmax(y)])
    seeds = list(S.WINDOW_SEEDS) + [f"vel:{lo}:1", f"angvel:{hi}:0"]
    R, dR = a.window_dual(T, seeds, 2)
    tgt = S.mse_target(R)
    gR = S.mse_grad(R, tgt)
    g = np.einsum("tgc,tgck->k", gR, dR)
    return R, tgt, g, (lo, hi), p


@pytest.mark.parametrize("k", range(6))
def test_dual_parameter_gradient_vs_central_differences(orc, dual_run, k):
    R, tgt, g, _, _ = dual_run
    group, key = S.WINDOW_PARAMS[k]
    base = {"normalK": 1e5, "shearK": 1e5, "torsionK": 1e5, "bendingK": 1e5, "viscosity": 1.0}[key]

    def loss_at(x):
        b = S.window_block(orc)
        b.set_group_param(group, key, x)
        return S.mse(S.wall_force_history(b, T), tgt)

    check_gradient(g[k], loss_at, base)


@pytest.mark.parametrize("k,field,c", [(6, "vel", 1), (7, "angvel", 0)])
def test_dual_velocity_gradient_vs_central_differences(orc, dual_run, k, field, c):
    """Initial velocity of the bonded particle nearest the bottom platen, initial spin of the
    bonded one nearest the top."""
    R, tgt, g, (lo, hi), p = dual_run
    pid = lo if field == "vel" else hi
    assert g[k] != 0.0
    v0, w0 = p["vel"], p["angvel"]   # rows by id, ids 0..n-1

    def loss_at(x):
        v, w = v0.copy(), w0.copy()
        (v if field == "vel" else w)[pid, c] = x
        return S.mse(S.wall_force_history(S.window_block(orc, vel=v, angvel=w), T), tgt)

    check_gradient(g[k], loss_at, (v0 if field == "vel" else w0)[pid, c])


# ---- bond failures inside the window: the forward's events, fixed for the derivative ----
BRK = dict(friction=True, strength=2000.0)   # ~20 of 184 bonds fail between steps 11 and 58


def test_dual_window_follows_bond_failures(orc):
    """Values equal the restatement's FP64 steps bit for bit through the failures (the
    failed bond leaves, its particles' new-list pairs join the friction group, the wall
    candidates are refreshed), and the failures happen inside the window."""
    a = S.window_block(orc, **BRK)
    R, dR = a.window_dual(T, list(S.WINDOW_SEEDS), 2)
    ref = S.wall_force_history(a, T)
    assert np.array_equal(R, ref)
    steps = a.breaks()[2]
    assert len(steps) >= 10 and steps.min() > 1 and steps.max() < T


@pytest.fixture(scope="module")
def dual_brk(orc):
    a = S.window_block(orc, **BRK)
    R, dR = a.window_dual(T, list(S.WINDOW_SEEDS), 2)
    tgt = S.mse_target(R)
    return tgt, np.einsum("tgc,tgck->k", S.mse_grad(R, tgt), dR)


# normalK, shearK, torsionK and the linear viscosity move the loss well above the rounding
# noise of a window with failing bonds and slipping contacts; bendingK and the rotational
# viscosity do not (their best central differences stay near 2e-4)
@pytest.mark.parametrize("k", [0, 1, 2, 4])
def test_dual_gradient_with_bond_failures_vs_central_differences(orc, dual_brk, k):
    tgt, g = dual_brk
    group, key = S.WINDOW_PARAMS[k]
    base = {"normalK": 1e5, "shearK": 1e5, "torsionK": 1e5, "viscosity": 1.0}[key]

    def loss_at(x):
        b = S.window_block(orc, **BRK)
        b.set_group_param(group, key, x)
        return S.mse(S.wall_force_history(b, T), tgt)

    check_gradient(g[k], loss_at, base)
