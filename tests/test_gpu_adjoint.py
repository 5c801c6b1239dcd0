"""Differentiable window on the GPU: reverse sweep vs the CPU dual-number window and
vs central finite differences of the GPU's own forward runs.  All tests need a GPU.

Bars: reactions within 1e-7 of the largest magnitude of the oracle's FP64 steps
(the two paths sum per-particle forces in different fixed orders and a loaded,
bouncing block amplifies last-bit differences over 200 steps); adjoint
gradients within 1e-5 relative of the dual-number derivatives of the same
window (same branches, exact derivatives of the same arithmetic); within 1e-4
relative of FP64 central differences at the best of h = 1e-6 ... 1e-2
relative; bit-identical gradients for any checkpoint interval.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

T = 200


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


@pytest.fixture(scope="module")
def orc(oracle_libs):
    return lambda *a: oracle_libs.OracleSim("orc", *a)


def _grad_vs(g_gpu, g_ref, rtol):
    scale = np.abs(g_ref)
    err = np.abs(g_gpu - g_ref)
    assert np.all(err <= rtol * scale + 1e-300), (g_gpu, g_ref, err / np.maximum(scale, 1e-300))


def _seed_particles(orc_sim):
    p = orc_sim.particles()
    i1, i2, _ = orc_sim.pairs("bonds")
    bonded = np.isin(p["id"], np.concatenate([i1, i2]))
    y = np.where(bonded, p["pos"][:, 1], np.nan)
    return int(p["id"][np.nanargmin(y)]), int(p["id"][np.nanargmax(y)])


@pytest.fixture(scope="module")
def block_run(gpu, orc):
    a = S.window_block(gpu)
    R = a.window_forward(T, 32)
    tgt = S.mse_target(R)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    b = S.window_block(orc)
    lo, hi = _seed_particles(b)
    Rd, dR = b.window_dual(T, list(S.WINDOW_SEEDS) + [f"vel:{lo}:1", f"angvel:{hi}:0"], 2)
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    return a, R, tgt, g, Rd, gd, (lo, hi)


def test_window_reactions_match_oracle(block_run):
    a, R, tgt, g, Rd, gd, _ = block_run
    assert R.shape == Rd.shape
    assert np.abs(R - Rd).max() <= 1e-7 * np.abs(Rd).max()


def test_adjoint_matches_dual_numbers(block_run):
    a, R, tgt, g, Rd, gd, (lo, hi) = block_run
    layout = a.param_layout()
    idx = [layout.index(k) for k in S.WINDOW_PARAMS]
    _grad_vs(g["params"][idx], gd[:6], 1e-5)
    _grad_vs(np.array([g["vel"][lo, 1], g["angvel"][hi, 0]]), gd[6:], 1e-5)


def _fd_best(loss_at, base, g, rtol=1e-4):
    errs = {}
    for rel in (1e-6, 1e-5, 1e-4, 1e-3, 1e-2):
        h = rel * max(abs(base), 1e-3)
        g_fd = (loss_at(base + h) - loss_at(base - h)) / (2 * h)
        errs[rel] = abs(g - g_fd) / abs(g_fd)
    assert min(errs.values()) <= rtol, (g, errs)


@pytest.mark.parametrize("k", range(6))
def test_adjoint_matches_central_differences(block_run, k):
    a, R, tgt, g, _, _, _ = block_run
    layout = a.param_layout()
    slot = layout.index(S.WINDOW_PARAMS[k])
    group, key = S.WINDOW_PARAMS[k]
    base = a.param_values()[slot]

    def loss_at(x):
        a.window_rewind()
        a.set_group_param(group, key, x)
        r = a.window_forward(T, 64)
        a.window_rewind()
        a.set_group_param(group, key, base)
        return S.mse(r, tgt)

    _fd_best(loss_at, base, g["params"][slot])


def test_initial_velocity_gradient_matches_central_differences(block_run):
    a, R, tgt, g, _, _, (lo, hi) = block_run
    a.window_rewind()
    p0 = a.particles()
    for field, pid, c in (("vel", lo, 1), ("angvel", hi, 0)):
        base = p0[field][pid, c]

        def loss_at(x):
            a.window_rewind()
            v = p0[field].copy()
            v[pid, c] = x
            a.set_particles(**{field: v}, id=p0["id"])
            r = a.window_forward(T, 64)
            a.window_rewind()
            a.set_particles(**{field: p0[field]}, id=p0["id"])
            return S.mse(r, tgt)

        _fd_best(loss_at, base, g[field][pid, c])


def test_checkpoint_interval_does_not_change_gradients(gpu):
    out = []
    for K in (1, 7, T):
        a = S.window_block(gpu)
        R = a.window_forward(T, K)
        tgt = S.mse_target(R)
        out.append(a.window_adjoint(S.mse_grad(R, tgt)))
    for o in out[1:]:
        for k in ("params", "vel", "angvel", "pos", "quat"):
            assert np.array_equal(o[k], out[0][k]), k


def test_rewind_reproduces_the_window(gpu):
    a = S.window_block(gpu)
    a.step(5)
    R1 = a.window_forward(80, 16)
    t1 = a.timestep
    p1 = a.particles()
    a.window_rewind()
    assert a.timestep == t1 - 80
    R2 = a.window_forward(80, 16)
    assert np.array_equal(R1, R2)
    p2 = a.particles()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(p1[k], p2[k]), k
    a.step(3)                      # the simulation carries on normally
    assert a.timestep == t1 + 3


def test_torch_window_function(gpu):
    import torch

    from esys.lsm.adjoint import DifferentiableWindow

    a = S.window_block(gpu)
    win = DifferentiableWindow(a, nsteps=60, checkpoint_every=16)
    theta = win.parameters().requires_grad_()
    v0, w0 = win.initial_velocities()
    v0.requires_grad_()
    R = win(theta, v0, w0)
    tgt = torch.from_numpy(S.mse_target(R.detach().numpy()))
    loss = ((R - tgt) ** 2).mean()
    loss.backward()
    # the same through the raw C ABI
    b = S.window_block(gpu)
    Rb = b.window_forward(60, 16)
    assert np.array_equal(Rb, R.detach().numpy())
    gb = b.window_adjoint(S.mse_grad(Rb, tgt.numpy()))
    # torch forms dLoss/dR by its own mean backward: equal to the last bits, so compare to 1e-10
    # of each output's scale
    assert np.abs(theta.grad.numpy() - gb["params"]).max() <= 1e-10 * np.abs(gb["params"]).max()
    assert np.abs(v0.grad.numpy() - gb["vel"]).max() <= 1e-10 * np.abs(gb["vel"]).max()
    # a second call rewinds to the window start: same reactions for the same inputs
    R2 = win(theta.detach(), v0.detach(), w0)
    assert torch.equal(R2, R.detach())


def test_window_refuses_a_bond_break(gpu):
    from esys.lsm._capi import DemError

    # bonds far weaker than their creation pre-stress: some break in the first step
    b = S.bonded_block(gpu, strength=(0.05, 0.1, 0.1, 0.05))
    with pytest.raises(DemError, match="bond broke"):
        b.window_forward(50, 10)
    t = b.timestep
    assert t >= 1
    b.step(2)                      # still usable, and the host clock followed the device
    assert b.timestep == t + 2


def test_friction_window_matches_dual_numbers(gpu, orc):
    """RotFriction contacts (with their tangential history) inside the window."""
    a = S.loaded_friction_pack(gpu)
    b = S.loaded_friction_pack(orc)
    a.step(20)
    b.step(20)
    n = 40
    R = a.window_forward(n, 8)
    tgt = S.mse_target(R)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    seeds = ["param:friction:normalK", "param:friction:shearK", "param:Damping:viscosity",
             "param:RotDamping:viscosity"]
    Rd, dR = b.window_dual(n, seeds, 2)
    assert np.abs(Rd).max() > 0 and np.abs(dR).max() > 0   # the walls carry load
    assert np.abs(R - Rd).max() <= 1e-9 * np.abs(Rd).max()
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    layout = a.param_layout()
    idx = [layout.index(k) for k in (("friction", "normalK"), ("friction", "shearK"), ("Damping", "viscosity"),
                                     ("RotDamping", "viscosity"))]
    _grad_vs(g["params"][idx], gd, 1e-6)


def test_elastic_nonrotational_window_matches_dual_numbers(gpu, orc):
    """NRotSphere packing: NRotElastic pairs, six walls, gravity and linear damping."""
    a = S.gravity_box(gpu, n_side=5)
    b = S.gravity_box(orc, n_side=5)
    a.step(50)
    b.step(50)
    n = 60
    R = a.window_forward(n, 16)
    tgt = S.mse_target(R)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    Rd, dR = b.window_dual(n, ["param:elastic:normalK", "param:Damping:viscosity"], 6)
    assert np.abs(R - Rd).max() <= 1e-9 * np.abs(Rd).max()
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    layout = a.param_layout()
    idx = [layout.index(("elastic", "normalK")), layout.index(("Damping", "viscosity"))]
    _grad_vs(g["params"][idx], gd, 1e-6)


def test_hand_written_bond_reverse_matches_dual_numbers(gpu):
    """The RotBond VJP in the reverse sweep (hand-written reverse of the law, the default)
    against the same VJP by forward-mode duals (6 tangents per pass)."""
    out = {}
    for nt in (0, 6):
        a = S.window_block(gpu)
        a.set_option("adjoint_bond_tangents", nt)
        R = a.window_forward(T, 32)
        tgt = S.mse_target(R)
        out[nt] = a.window_adjoint(S.mse_grad(R, tgt))
    for k in ("params", "vel", "angvel", "pos", "quat"):
        scale = np.abs(out[6][k]).max()
        assert np.abs(out[0][k] - out[6][k]).max() <= 1e-9 * scale, k


# ---- bond failures inside the window (device bond hand-off) ----
BRK = dict(friction=True, strength=2000.0)   # ~20 of 184 bonds fail between steps 11 and 58


def _breaking(gpu):
    a = S.window_block(gpu, **BRK)
    a.set_option("bond_handoff", 1)
    return a


@pytest.fixture(scope="module")
def brk_run(gpu, orc):
    a = _breaking(gpu)
    R = a.window_forward(T, 32)
    ev = a.breaks()
    tgt = S.mse_target(R)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    b = S.window_block(orc, **BRK)
    lo, hi = _seed_particles(b)
    Rd, dR = b.window_dual(T, list(S.WINDOW_SEEDS) + [f"vel:{lo}:1", f"angvel:{hi}:0"], 2)
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    c = S.window_block(orc, **BRK)
    c.step(T)
    return a, R, ev, tgt, g, Rd, gd, c.breaks(), (lo, hi)


def test_window_with_bond_failures_matches_oracle(brk_run):
    a, R, ev, tgt, g, Rd, gd, ev_orc, _ = brk_run
    assert len(ev[0]) >= 10
    for u, v in zip(ev, ev_orc):
        assert np.array_equal(u, v)
    assert np.abs(R - Rd).max() <= 1e-7 * np.abs(Rd).max()


def test_adjoint_with_bond_failures_matches_dual_numbers(brk_run):
    a, R, ev, tgt, g, Rd, gd, _, (lo, hi) = brk_run
    layout = a.param_layout()
    idx = [layout.index(k) for k in S.WINDOW_PARAMS]
    _grad_vs(g["params"][idx], gd[:6], 1e-5)
    _grad_vs(np.array([g["vel"][lo, 1], g["angvel"][hi, 0]]), gd[6:], 1e-5)


def test_bond_failures_checkpoint_interval_does_not_change_gradients(gpu):
    """The recompute replays the failures (wall candidacy and last-failure record restored
    per segment), so segments of 1 step and one segment of the whole window agree."""
    out = []
    for K in (1, 13, T):
        a = _breaking(gpu)
        R = a.window_forward(T, K)
        tgt = S.mse_target(R)
        out.append(a.window_adjoint(S.mse_grad(R, tgt)))
        assert len(a.breaks()[0]) >= 10       # the recompute logged nothing again
    for o in out[1:]:
        for k in ("params", "vel", "angvel", "pos", "quat"):
            assert np.array_equal(o[k], out[0][k]), k


def test_rewind_undoes_bond_failures(gpu):
    a = _breaking(gpu)
    R1 = a.window_forward(T, 40)
    e1 = a.breaks()
    p1 = a.particles()
    a.window_rewind()
    assert len(a.breaks()[0]) == 0
    R2 = a.window_forward(T, 40)
    assert np.array_equal(R1, R2)
    for u, v in zip(e1, a.breaks()):
        assert np.array_equal(u, v)
    p2 = a.particles()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(p1[k], p2[k]), k
    a.step(5)                      # the failures are handed on to the ordinary stepping
    assert a.timestep == T + 5


# ---- the window in the FP32-force form ----
def test_fp32_form_window_matches_fp64_dual_numbers(gpu, orc):
    """FP32 pair forces in the forward and its recompute (RotFriction contacts and RotBonds,
    bonds failing inside the window under the hand-off); the reverse linearises each law in
    FP64 at the FP32 trajectory.  Bar: 1e-4 relative of the FP64 dual-number derivatives,
    the spec's bar against FP64 differences."""
    a = _breaking(gpu)
    a.set_option("precision", 32)
    R = a.window_forward(T, 32)
    b = S.window_block(orc, **BRK)
    lo, hi = _seed_particles(b)
    Rd, dR = b.window_dual(T, list(S.WINDOW_SEEDS) + [f"vel:{lo}:1", f"angvel:{hi}:0"], 2)
    # the FP32 forces move the reactions by ~1e-7 of their scale
    assert np.abs(R - Rd).max() <= 1e-5 * np.abs(Rd).max()
    tgt = S.mse_target(Rd)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    layout = a.param_layout()
    idx = [layout.index(k) for k in S.WINDOW_PARAMS]
    _grad_vs(g["params"][idx], gd[:6], 1e-4)
    _grad_vs(np.array([g["vel"][lo, 1], g["angvel"][hi, 0]]), gd[6:], 1e-4)


def test_fp32_form_window_checkpoints_and_rewind(gpu):
    out = []
    for K in (1, T):
        a = _breaking(gpu)
        a.set_option("precision", 32)
        R = a.window_forward(T, K)
        tgt = S.mse_target(R)
        out.append(a.window_adjoint(S.mse_grad(R, tgt)))
        a.window_rewind()
        assert np.array_equal(a.window_forward(T, K), R)
    for k in ("params", "vel", "angvel"):
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("case", ["friction", "elastic", "bonded_failing"])
def test_hand_written_pair_reverse_matches_dual_numbers(gpu, case):
    """The RotFriction and NRotElastic VJPs of the reverse sweep (hand-written reverses, the
    default) against the same VJPs by forward-mode duals."""
    out = {}
    for duals in (0, 1):
        if case == "friction":
            a = S.loaded_friction_pack(gpu)
            a.step(20)
            n, ng = 40, 2
        elif case == "elastic":
            a = S.gravity_box(gpu, n_side=5)
            a.step(50)
            n, ng = 60, 6
        else:
            a = _breaking(gpu)
            n, ng = T, 2
        a.set_option("adjoint_pair_duals", duals)
        R = a.window_forward(n, 16)
        tgt = S.mse_target(R)
        out[duals] = a.window_adjoint(S.mse_grad(R, tgt))
    for k in ("params", "vel", "angvel", "pos"):
        scale = np.abs(out[1][k]).max()
        assert scale > 0 or k == "angvel", k
        assert np.abs(out[0][k] - out[1][k]).max() <= 1e-10 * max(scale, 1e-300), k


def test_fitted_polydisperse_window_matches_dual_numbers(gpu, orc):
    """The bench's window at 2,000 spheres (radii 0.2 to 1.0, fitted packing). On it, central
    differences of the torsion / bending stiffness and the rotational viscosity do not settle (the
    loss is rough in them at every step size from 1e-3 to 2e-2 relative), while the normal
    stiffness's do; the GPU reverse equals the CPU restatement's forward-mode derivative, which
    is exact for the computed trajectory, on all of them."""
    T = 300
    a = S.fitted_window_block(gpu)
    R = a.window_forward(T, 50)
    tgt = S.mse_target(R)
    g = a.window_adjoint(S.mse_grad(R, tgt))
    b = S.fitted_window_block(orc)
    keys = [("bonds", "normalK"), ("bonds", "torsionK"), ("bonds", "bendingK"), ("RotDamping", "viscosity"),
            ("Damping", "viscosity")]
    Rd, dR = b.window_dual(T, [f"param:{grp}:{k}" for grp, k in keys], 2)
    assert np.abs(R - Rd).max() <= 1e-7 * np.abs(Rd).max()
    gd = np.einsum("tgc,tgck->k", S.mse_grad(Rd, tgt), dR)
    layout = a.param_layout()
    _grad_vs(g["params"][[layout.index(k) for k in keys]], gd, 1e-4)
