"""Benchmark of the B200 DEM step on the rotational frictional shear cell, with legs for the
other workloads of the per-timestep hot path.

Headline workload: 250,000 RotSpheres, lognormal radii (median 0.5, sigma 0.25, clipped to
[0.2, 1.0]) packed by seeded random sequential insertion into a 100 x 50 x 100 box periodic
in x; RotFriction kn = ks = 1e4, mu = 0.6; elastic walls (k = 1e4) at y = 0 and y = 50 moving
at -/+0.01 in x with a 1e3 normal-load servo on the top wall; dt = 5e-5.  Initial velocities
and spins are seeded N(0, 0.1) so that contacts form.

One bench "step" = --dem-steps timesteps (runOneStep x S) plus one servo call.  `value` is
contact-updates/s (Verlet-list pairs + wall candidates evaluated per timestep) with the state
resident in HBM; `e2e` repeats it through the C ABI with the particle state copied
host->device before and device->host after every bench step.  L2 is flushed between bench
steps.  Legs: the 8,000-sphere gravity packing (FP64), the 1,000,000-sphere bonded block
(FP32-force and FP64 forms), the NRotFriction law on the headline packing, the
differentiable calibration window and the batched ensemble of bonded cylinders, each beside
the reference's own C++ timed on this host's cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "esys-particle_b200"))

PI_REF = 3.141592654
METRIC = "contact-updates/s at <=1e-5 rel force err vs FP64"
UNIT = "contact-updates/s"


def _jsonable(o):
    """numpy scalars and arrays in the JSON line as plain numbers and lists."""
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError(f"{type(o).__name__} is not JSON serializable")


def product_rsi(seed, n, bmin, bmax, periodic_x, dist, p0, p1, rmin, rmax, max_attempts):
    """The seeded RSI packer of the product library (include/esys_geometry.h)."""
    from esys.lsm import geometry as G

    kw = {"lognormal": (p0, p1)} if dist == 1 else {"uniform": (p0, p1)}
    return G.rsi_pack(n, bmin, bmax, seed=seed, periodic_x=bool(periodic_x), rmin=rmin, rmax=rmax,
                      max_attempts=max_attempts, **kw)


def workload(n=250_000, seed=2, packer=None):
    """Seeded shear-cell packing.  `packer` is the RSI packer to use (the product library's by
    default; the reference arm passes the same packer linked into the reference library, so it
    loads no product code): both give the same spheres for the same seed."""
    packer = packer or product_rsi
    bmin = np.array([0.0, 0.0, 0.0])
    bmax = np.array([100.0, 50.0, 100.0])
    pos, rad = packer(seed, n, bmin, bmax, 1, 1, 0.5, 0.25, 0.2, 1.0, 5000)
    if len(rad) != n:
        raise RuntimeError(f"packer placed {len(rad)} of {n} spheres")
    rng = np.random.default_rng(seed + 100)
    vel = rng.normal(0.0, 0.1, size=(n, 3))
    angvel = rng.normal(0.0, 0.1, size=(n, 3))
    mass = (4.0 / 3.0) * 1.0 * PI_REF * rad * rad * rad
    return dict(pos=pos, rad=rad, mass=mass, vel=vel, angvel=angvel, bmin=bmin, bmax=bmax,
                ids=np.arange(n, dtype=np.int32))


HEADLINE_WORKLOAD = ("rot-friction shear cell: 250,000 RotSpheres, lognormal r (0.5, 0.25) in [0.2,1.0], 100x50x100, "
                     "kn=ks=1e4 mu=0.6, 2 elastic walls +-0.01 x, 1e3 servo load, dt=5e-5")
DT = 5e-5
GRID, SKIN = 2.2, 0.2
KN = KS = 1e4
MU = 0.6
KWALL = 1e4
NORMAL_LOAD = 1e3


def setup(make, w, periodic=True):
    sim = make("RotSphere", GRID, SKIN, w["bmin"], w["bmax"], (1 if periodic else 0, 0, 0), DT)
    sim.add_particles(w["ids"], w["pos"], w["rad"], w["mass"], tag=np.zeros(len(w["ids"]), np.int32),
                      vel=w["vel"], angvel=w["angvel"])
    sim.add_rot_friction_group("friction", KN, MU, MU, KS, DT, True, True)
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, 50, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", KWALL)
    sim.add_wall_group("top_w", "top", KWALL)
    return sim


class Clocks:
    """Sample SM clocks, power and throttle reasons during the timed region.

    Through NVML in-process (the library nvidia-smi reads), on the GPU this process runs on
    (matched by UUID): spawning nvidia-smi from a thread forks a process that holds a large
    CUDA context, and those forks stalled the timed host loop.  nvidia-smi is the fallback."""

    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, index=0):
        self.samples, self._stop, self.index = [], False, index

    def _nvml(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

        def sample():
            sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
            pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
            bits = int(reasons(h))
            return [sm, mx, pw, bits]

        return sample

    def __enter__(self):
        try:
            sample = self._nvml()
        except Exception:
            sample = None
        self.source = "nvml" if sample is not None else "nvidia-smi"

        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop:
                try:
                    if sample is not None:
                        self.samples.append(sample())
                    else:
                        out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                             timeout=5).stdout.strip()
                        if out:
                            v = [x.strip() for x in out.split(",")]
                            bits = sum(b for b, k in zip((0x8, 0x40, 0x20, 0x4), v[3:7]) if k == "Active")
                            self.samples.append([float(v[0]), float(v[1]), float(v[2]), bits])
                except Exception:
                    pass
                time.sleep(0.05 if sample is not None else 0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop = True
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        mx = [s[1] for s in self.samples]
        reasons = sorted({name for s in self.samples for bit, name in self.REASONS.items() if s[3] & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": reasons,
                "samples": len(self.samples), "power_w_median": float(np.median([s[2] for s in self.samples])),
                "source": self.source}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch():
    p = os.path.join(ROOT, "profiles", "k_step_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


def cpu_reference_sample(w, steps, timeout_s=60.0):
    """The reference's own C++ (oracle/_ref, one worker = one core) on the same packing.
    The reference reaches periodic x only with >= 2 MPI workers, so the sample runs it with
    the same particles and groups in a non-periodic box."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.available("ref"):
        return None
    sim = setup(lambda *a: oracle.OracleSim("ref", *a), w, periodic=False)
    sim.step(1)  # first step: neighbour search + interaction set-up (not timed)
    m = sim.f["num_pairs"](sim.h, b"friction")
    pos = w["pos"]
    ncand = int((np.abs(pos[:, 1] - 0.0) < GRID).sum() + (np.abs(pos[:, 1] - 50.0) < GRID).sum())
    done, t0 = 0, time.perf_counter()
    while done < steps and time.perf_counter() - t0 < timeout_s:
        sim.step(1)
        done += 1
    dt = time.perf_counter() - t0
    return {"value": (m + ncand) * done / dt, "steps": done, "seconds": dt, "pairs": int(m), "walls": ncand}


# ---- differentiable calibration window (adjoint leg) --------------------------------------
W_DT, W_STEPS, W_CKPT = 1e-5, 2000, 100
W_KN, W_KS, W_KT, W_KB, W_VISC = 1e5, 1e5, 1e3, 1e3, 0.05


def window_workload(n=50_000, seed=4):
    """Bonded block: n RotSpheres fitted into 40 x 80 x 40 (radii in [0.2, 1.0]), every pair
    within a 1e-3 gap bonded; seeded small initial velocities."""
    from esys.lsm import geometry as G

    pos, rad = G.fit_pack(n, (0, 0, 0), (40, 80, 40), 0.2, 1.0, seed=seed, max_failures=5000)
    i1, i2 = G.distance_connections(pos, rad, 1e-3)
    rng = np.random.default_rng(seed + 100)
    m = len(rad)
    return dict(pos=pos, rad=rad, mass=(4.0 / 3.0) * PI_REF * rad ** 3, ids=np.arange(m, dtype=np.int32),
                vel=rng.normal(0, 0.01, size=(m, 3)), angvel=rng.normal(0, 0.01, size=(m, 3)), i1=i1, i2=i2)


def window_setup(make, w):
    sim = make("RotSphere", 2.2, 0.2, (0, 0, 0), (40, 80, 40), (0, 0, 0), W_DT)
    n = len(w["ids"])
    sim.add_particles(w["ids"], w["pos"], w["rad"], w["mass"], tag=np.zeros(n, np.int32), vel=w["vel"],
                      angvel=w["angvel"])
    sim.add_connections(np.ones(len(w["i1"]), np.int32), w["i1"], w["i2"])
    sim.add_rot_bond_group("bonds", 1, W_KN, W_KS, W_KT, W_KB, 1e6, 1e6, 1e6, 1e6, True, True, 1.0)
    y0 = float((w["pos"][:, 1] - w["rad"]).min())
    y1 = float((w["pos"][:, 1] + w["rad"]).max())
    sim.add_wall("bottom", (0, y0, 0), (0, 1, 0))
    sim.add_wall("top", (0, y1, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, W_VISC, 100)
    sim.add_damping(1, W_VISC, 100)
    sim.set_wall_velocity("bottom", (0, 1.0, 0))
    sim.set_wall_velocity("top", (0, -1.0, 0))
    return sim


def window_target(R, seed=4):
    """Seeded target curve: a smooth ramp per platen with the window's own scale."""
    rng = np.random.default_rng(seed)
    t = np.linspace(0.0, 1.0, R.shape[0])[:, None, None]
    return np.abs(R).max() * rng.uniform(0.5, 1.0, size=(1, R.shape[1], 3)) * t * np.sign(R.mean(axis=0) + 1e-300)


def adjoint_leg(stream, precision=32):
    """Forward window + reverse sweep on the C4-style bonded block in the FP32-force form (FP32
    pair forces in the forward and its recompute, FP64 reverse); adjoint grads/s vs the
    central-difference alternative (two forward windows per gradient component), and the
    adjoint gradients of kn, ks, kt, kb, the linear and rotational damping and three initial
    velocity components against FP64 central differences (h = 1e-6 relative; the best of
    h = 1e-6, 1e-5, 1e-4 is reported beside it, as a 2,000-step loaded window carries FP64
    rounding noise in its loss)."""
    from esys.lsm import _capi

    w = window_workload()
    sim = window_setup(lambda *a: _capi.DemSim(*a), w)
    sim.set_stream(stream.cuda_stream)
    sim.set_option("precision", precision)
    sim.step(1)  # set-up step (first neighbour search), not part of the window
    n = sim.num_particles()
    t0 = time.perf_counter()
    R = sim.window_forward(W_STEPS, W_CKPT)
    t1 = time.perf_counter()
    tgt = window_target(R)
    gR = 2.0 * (R - tgt) / R.size
    g = sim.window_adjoint(gR)
    t2 = time.perf_counter()
    loss0 = float(((R - tgt) ** 2).mean())
    sim.window_rewind()
    t3 = time.perf_counter()
    sim.window_forward(W_STEPS, W_STEPS)  # a plain forward window: the unit cost of a difference
    t4 = time.perf_counter()
    layout = sim.param_layout()
    sim.close()

    # FP64 central differences on a second handle of the same block
    ref = window_setup(lambda *a: _capi.DemSim(*a), w)
    ref.set_stream(stream.cuda_stream)
    ref.set_option("precision", 64)
    ref.step(1)
    # the FP64 form's own adjoint of the same window, beside the FP32 form's
    R64 = ref.window_forward(W_STEPS, W_CKPT)
    g64 = ref.window_adjoint(2.0 * (R64 - tgt) / R64.size)
    ref.window_rewind()
    p0 = ref.particles()
    base_vals = ref.param_values()
    loss_base = float(((R64 - tgt) ** 2).mean())

    def mse(r):
        return float(((r - tgt) ** 2).mean())

    def loss_param(slot, x):
        group, key = ref.param_layout()[slot]
        ref.window_rewind()
        ref.set_group_param(group, key, x)
        r = ref.window_forward(W_STEPS, W_STEPS)
        ref.window_rewind()
        ref.set_group_param(group, key, base_vals[slot])
        return mse(r)

    def loss_vel(row, c, x):
        ref.window_rewind()
        v = p0["vel"].copy()
        v[row, c] = x
        ref.set_particles(vel=v, id=p0["id"])
        r = ref.window_forward(W_STEPS, W_STEPS)
        ref.window_rewind()
        ref.set_particles(vel=p0["vel"], id=p0["id"])
        return mse(r)

    def central(f, base, g_adj, g_adj64):
        """Central differences at h = 1e-6 ... 1e-2 relative.  The second difference
        |L(x+h) + L(x-h) - 2 L(x)| bounds the loss's rounding noise at that h (its curvature term
        is far smaller); a difference is resolved when it exceeds 100x that noise over 2h."""
        rows = {}
        for rel in (1e-6, 1e-5, 1e-4, 1e-3, 1e-2):
            h = rel * max(abs(base), 1e-12)
            lp, lm = f(base + h), f(base - h)
            fd = (lp - lm) / (2 * h)
            noise = abs(lp + lm - 2.0 * loss_base) / (2 * h)
            rows[rel] = {"fd": float(fd), "noise": float(noise), "resolved": bool(abs(fd) > 100.0 * noise),
                         "rel_err": float(abs(g_adj - fd) / max(abs(fd), 1e-300)),
                         "rel_err_fp64_adjoint": float(abs(g_adj64 - fd) / max(abs(fd), 1e-300))}
        res = [r for r in rows.values() if r["resolved"]] or list(rows.values())
        best = min(res, key=lambda r: r["rel_err"])
        return {"adjoint": float(g_adj), "adjoint_fp64": float(g_adj64), "central_difference": rows[1e-6]["fd"],
                "rel_err": rows[1e-6]["rel_err"], "resolved_at_1e-6": rows[1e-6]["resolved"],
                "best_rel_err": best["rel_err"], "best_rel_err_fp64_adjoint": min(r["rel_err_fp64_adjoint"] for r in res),
                "resolved_h_rel": [k for k, r in rows.items() if r["resolved"]]}

    checks = {}
    for group, key in (("bonds", "normalK"), ("bonds", "shearK"), ("bonds", "torsionK"), ("bonds", "bendingK"),
                       ("Damping", "viscosity"), ("RotDamping", "viscosity")):
        slot = layout.index((group, key))
        checks[f"{group}.{key}"] = central(lambda x, s_=slot: loss_param(s_, x), base_vals[slot], g["params"][slot],
                                           g64["params"][slot])
    # the three initial velocity components the loss depends on most (rows sorted by id)
    gv = g["vel"]
    for flat in np.argsort(-np.abs(gv).ravel())[:3]:
        row, c = divmod(int(flat), 3)
        checks[f"vel[id {int(p0['id'][row])}][{'xyz'[c]}]"] = central(
            lambda x, r_=row, c_=c: loss_vel(r_, c_, x), p0["vel"][row, c], gv[row, c], g64["vel"][row, c])
    ref.close()
    grads = len(g["params"]) + 3 * n  # parameters and initial linear velocities (spins come too, uncounted)
    t_adj = t2 - t0
    t_fwd = t4 - t3
    bonds = len(w["i1"])
    return {
        "workload": f"bonded block: {n} RotSpheres fitted in 40x80x40 (r in [0.2,1.0]), {bonds} RotBonds "
                    f"(kn=ks=1e5, kt=kb=1e3, elastic regime), 2 elastic platens at 1.0/s, linear+rotational "
                    f"damping 0.05, dt=1e-5, {W_STEPS}-step window, checkpoints every {W_CKPT}",
        "loss": "MSE of the platen reaction histories vs a seeded ramp target", "loss_value": loss0,
        "dtype": ("f32-forces/f64-integration forward and recompute, f64 reverse" if precision == 32 else "f64"),
        "gradient_components": grads,
        "forward_with_checkpoints_s": t1 - t0, "reverse_sweep_s": t2 - t1, "plain_forward_s": t_fwd,
        "adjoint_grads_per_s": grads / t_adj, "fd_grads_per_s": 1.0 / (2.0 * t_fwd),
        "adjoint_vs_fd_speedup": (grads / t_adj) / (1.0 / (2.0 * t_fwd)),
        "fd_checks": checks,
        "fd_max_rel_err_resolved_1e-6": max([c["rel_err"] for c in checks.values() if c["resolved_at_1e-6"]],
                                            default=None),
        "fd_max_best_rel_err": max(c["best_rel_err"] for c in checks.values()),
        "fd_max_best_rel_err_fp64_adjoint": max(c["best_rel_err_fp64_adjoint"] for c in checks.values()),
    }


# ---- batched ensemble leg ------------------------------------------------------------------
E_DT = 1e-5
E_RHO = 2.2  # spheres per unit volume of the fitting packer (radii in [0.2, 1.0], 300 failures)


def specimen_target_count(k, seed=5):
    """The particle count specimen k aims at (its first seeded draw)."""
    return float(np.exp(np.random.default_rng(seed + k).uniform(np.log(2000), np.log(40000))))


def cylinder_specimen(k, seed=5):
    """Specimen k: a bonded cylinder (height 4R) cut from a fitting-packer block, its particle
    count log-uniform in [2,000, 40,000]; bond stiffness and strengths log-uniform."""
    from esys.lsm import geometry as G

    rng = np.random.default_rng(seed + k)
    n_t = float(np.exp(rng.uniform(np.log(2000), np.log(40000))))
    R = (n_t / (E_RHO * 4.0 * np.pi)) ** (1.0 / 3.0)
    H = 4.0 * R
    pos, rad = G.fit_pack(int(2 * n_t) + 100, (-R, 0, -R), (R, H, R), 0.2, 1.0, seed=seed * 1000 + k,
                          max_failures=300)
    keep = pos[:, 0] ** 2 + pos[:, 2] ** 2 <= R * R
    pos, rad = pos[keep], rad[keep]
    i1, i2 = G.distance_connections(pos, rad, 1e-3)
    kn, ks = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=2))
    sn, ss = np.exp(rng.uniform(np.log(0.1), np.log(2.0), size=2))
    m = len(rad)
    return dict(n=m, pos=pos, rad=rad, i1=i1, i2=i2, R=R, H=H, kn=kn, ks=ks, sn=sn, ss=ss,
                vel=np.zeros((m, 3)), angvel=np.zeros((m, 3)))


def cylinder_sim(make, sp, grid=2.2, skin=0.2):
    """Per specimen as the bonded-block compression: RotBond (kt = kb = 1e3, torsion / bending
    strengths = shear / normal), RotFriction for post-break contacts with the bond exclusion,
    elastic platens closing by 1e-7 of the height per step (the bonded-block compression rate:
    1e-4 x 200 / 1000 per step on a height of 200), light damping; at rest initially."""
    R, H = sp["R"], sp["H"]
    sim = make("RotSphere", grid, skin, (-R - 1, -1, -R - 1), (R + 1, H + 1, R + 1), (0, 0, 0), E_DT)
    n = sp["n"]
    sim.add_particles(np.arange(n, dtype=np.int32), sp["pos"], sp["rad"], (4.0 / 3.0) * PI_REF * sp["rad"] ** 3,
                      tag=np.zeros(n, np.int32), vel=sp["vel"], angvel=sp["angvel"])
    sim.add_connections(np.ones(len(sp["i1"]), np.int32), sp["i1"], sp["i2"])
    sim.add_rot_bond_group("bonds", 1, sp["kn"], sp["ks"], 1e3, 1e3, sp["sn"], sp["ss"], sp["ss"], sp["sn"],
                           True, True, 1.0)
    sim.add_rot_friction_group("friction", sp["kn"], 0.6, 0.6, sp["ks"], E_DT, True, True)
    sim.add_exclusion("bonds", "friction")
    y0 = float((sp["pos"][:, 1] - sp["rad"]).min())
    y1 = float((sp["pos"][:, 1] + sp["rad"]).max())
    sim.add_wall("bottom", (0, y0, 0), (0, 1, 0))
    sim.add_wall("top", (0, y1, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, 0.01, 100)
    sim.add_damping(1, 0.01, 100)
    v = 0.5 * 1e-7 * H / E_DT
    sim.set_wall_velocity("bottom", (0, v, 0))
    sim.set_wall_velocity("top", (0, -v, 0))
    sim.set_option("bond_handoff", 1)
    return sim


def nrot_friction_leg(stream, steps=1000, ref_steps=20):
    """The widened pair law on the headline packing: the 250,000 spheres as NRotSpheres with an
    NRotFriction group (CFrictionInteraction, k = ks = 1e4, mu = 0.6), the elastic walls moving
    at -+0.01 in x; the GPU's FP64 form (the law's only form) against the reference's own C++
    (oracle/_ref, one core, non-periodic as for the headline's baseline)."""
    import torch

    from esys.lsm import _capi

    w = workload()

    def build(make, periodic):
        sim = make("NRotSphere", GRID, SKIN, w["bmin"], w["bmax"], (1 if periodic else 0, 0, 0), DT)
        sim.add_particles(w["ids"], w["pos"], w["rad"], w["mass"], tag=np.zeros(len(w["ids"]), np.int32),
                          vel=w["vel"])
        sim.add_nrot_friction_group("friction", KN, MU, KS, DT, True)
        sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
        sim.add_wall("top", (0, 50, 0), (0, -1, 0))
        sim.add_wall_group("bottom_w", "bottom", KWALL)
        sim.add_wall_group("top_w", "top", KWALL)
        return sim

    sim = build(lambda *a: _capi.DemSim(*a), True)
    sim.set_stream(stream.cuda_stream)
    sim.set_option("profile", 1)
    sim.set_wall_velocity("bottom", (-0.01, 0, 0))
    sim.set_wall_velocity("top", (0.01, 0, 0))
    sim.step(200)
    torch.cuda.synchronize()
    c0 = sim.counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    c1 = sim.counters()
    ms = e0.elapsed_time(e1)
    value = (c1["contact_updates"] - c0["contact_updates"]) / (ms / 1e3)
    kus = (c1["step_kernel_ns"] - c0["step_kernel_ns"]) / max(1, c1["profiled_steps"] - c0["profiled_steps"]) / 1e3
    touching = int(sim.pairs("friction")[2][:, 4].sum())
    sim.close()
    ref = None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if oracle.available("ref"):
        r = build(lambda *a: oracle.OracleSim("ref", *a), False)
        r.step(1)
        m = r.f["num_pairs"](r.h, b"friction")
        ncand = int((np.abs(w["pos"][:, 1]) < GRID).sum() + (np.abs(w["pos"][:, 1] - 50.0) < GRID).sum())
        t0 = time.perf_counter()
        r.step(ref_steps)
        dt = time.perf_counter() - t0
        ref = {"value": (m + ncand) * ref_steps / dt, "steps": ref_steps, "cores": 1, "kind": "reference"}
    return {
        "workload": "the headline's 250,000-sphere packing as NRotSpheres, NRotFriction k=ks=1e4 mu=0.6, "
                    "2 elastic walls -+0.01 x, dt=5e-5",
        "metric": "contact-updates/s", "value": value, "steps": steps, "dtype": "f64", "kernel_us": kus,
        "touching_pairs": touching, "cpu_reference": ref,
        "speedup_vs_cpu_reference": value / ref["value"] if ref else None,
    }


# ---- gravity packing (8,000 NRotSpheres, FP64) --------------------------------------------
G_DT, G_STEPS = 1e-4, 5000


def gravity_world(n_side=20, layers=20, seed=1):
    """8,000 NRotSpheres on a 20 x 20 x 20 cubic lattice (spacing 1, jitter U(-0.05, 0.05)) in
    the lower half of a 20 x 20 x 40 box, radii U[0.4, 0.5], density 1."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(layers), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) + rng.uniform(-0.05, 0.05, size=g.shape)
    rad = rng.uniform(0.4, 0.5, size=len(g))
    return dict(pos=pos, rad=rad, L=float(n_side), H=2.0 * layers)


def gravity_sim(make, w):
    """NRotElastic k = 1000 (scaled), gravity -9.81 z, linear damping 0.01, six elastic walls
    k = 1000 on the box faces; gridSpacing 1.2, verletDist 0.2, dt = 1e-4."""
    L, H = w["L"], w["H"]
    n = len(w["rad"])
    sim = make("NRotSphere", 1.2, 0.2, (0, 0, 0), (L, L, H), (0, 0, 0), G_DT)
    sim.add_particles(np.arange(n, dtype=np.int32), w["pos"], w["rad"], (4.0 / 3.0) * PI_REF * w["rad"] ** 3,
                      tag=np.zeros(n, np.int32))
    sim.add_elastic_group("elastic", 1000.0, True)
    sim.add_gravity("gravity", (0, 0, -9.81))
    sim.add_damping(0, 0.01, 100)
    for name, o, nrm in (("xlo", (0, 0, 0), (1, 0, 0)), ("xhi", (L, 0, 0), (-1, 0, 0)),
                         ("ylo", (0, 0, 0), (0, 1, 0)), ("yhi", (0, L, 0), (0, -1, 0)),
                         ("zlo", (0, 0, 0), (0, 0, 1)), ("zhi", (0, 0, H), (0, 0, -1))):
        sim.add_wall(name, o, nrm)
        sim.add_wall_group(name + "_w", name, 1000.0)
    return sim


def timed_run(sim, stream, steps):
    """steps timesteps of a library handle on `stream`, timed with CUDA events; returns the
    device milliseconds and the handle's counters before and after."""
    import torch

    torch.cuda.synchronize()
    c0 = sim.counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), c0, sim.counters()


def cpu_sample(sim, budget_s, max_steps, before=None):
    """Timesteps of a CPU harness within a time budget (after its first, set-up step);
    `before` runs ahead of every timestep (a pre-step runnable)."""
    if before:
        before()
    sim.step(1)
    done, t0 = 0, time.perf_counter()
    while done < max_steps and time.perf_counter() - t0 < budget_s:
        if before:
            before()
        sim.step(1)
        done += 1
    return done, time.perf_counter() - t0


def gravity_leg(stream, cpu=True, cpu_budget=20.0):
    """The plain-FP64 gravity packing over its full 5,000 steps on the GPU, beside the
    reference's own C++ (one core) on the same spheres."""
    from esys.lsm import _capi

    w = gravity_world()
    sim = gravity_sim(lambda *a: _capi.DemSim(*a), w)
    sim.set_stream(stream.cuda_stream)
    sim.set_option("profile", 1)
    sim.set_option("precision", 64)
    sim.step(1)  # set-up: first neighbour search
    ms, c0, c1 = timed_run(sim, stream, G_STEPS)
    n = len(w["rad"])
    cu = c1["contact_updates"] - c0["contact_updates"]
    kus = (c1["step_kernel_ns"] - c0["step_kernel_ns"]) / max(1, c1["profiled_steps"] - c0["profiled_steps"]) / 1e3
    m = len(sim.pairs("elastic")[0])
    touching = int(np.sum(sim.interaction_scalar_field("elastic", "count")[2]))
    walls = c1["contacts_per_step"] - m
    alg = n * 136 + m * 8 + walls * 4
    sim.close()
    out = {
        "workload": "gravity packing: 8,000 NRotSpheres (20x20x20 jittered lattice, r in [0.4,0.5]) in a 20x20x40 "
                    "box, NRotElastic k=1000, gravity -9.81 z, linear damping 0.01, 6 elastic walls k=1000, dt=1e-4",
        "metric": "contact-updates/s", "value": cu / (ms / 1e3), "dtype": "f64", "timesteps": G_STEPS,
        "timesteps_per_s": G_STEPS / (ms / 1e3), "ms_total": ms, "kernel_us": kus,
        "elastic_pairs": m, "wall_candidates": walls, "touching_pairs_end": touching,
        "roofline": {"bound": "hbm", "achieved_gbs": alg / (kus * 1e-6) / 1e9 if kus > 0 else None,
                     "algorithmic_bytes_per_timestep": alg,
                     "note": "8,000 spheres: the step is launch- and latency-bound, far below HBM bandwidth"},
        "cpu_reference": None,
    }
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        if oracle.available("ref"):
            r = gravity_sim(lambda *a: oracle.OracleSim("ref", *a), w)
            done, dt = cpu_sample(r, cpu_budget, G_STEPS)
            m_r = r.f["num_pairs"](r.h, b"elastic")
            out["cpu_reference"] = {"value": (m_r + walls) * done / dt, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"{done} of the {G_STEPS} timesteps after set-up"}
            out["speedup_vs_cpu_reference"] = out["value"] / out["cpu_reference"]["value"]
    return out


# ---- bonded block (1,000,000 RotSpheres) ------------------------------------------------------
B_DT = 1e-5


def block_world(n=1_000_000, seed=3):
    """The fitting packer's 1M spheres (radii in [0.2, 1.0]) in 66 x 132 x 66 (the 100 x 200 x 100
    prism of the spec holds 1M spheres only at uniform radii), every pair within a 1e-3 gap bonded.
    Another n scales the box by (n / 1M)^(1/3) at the same packing density."""
    from esys.lsm import geometry as G

    f = (n / 1e6) ** (1.0 / 3.0)
    box = (66 * f, 132 * f, 66 * f)
    pos, rad = G.fit_pack(n, (0, 0, 0), box, 0.2, 1.0, seed=seed, max_failures=300)
    i1, i2 = G.distance_connections(pos, rad, 1e-3)
    return dict(pos=pos, rad=rad, i1=i1, i2=i2, box=box)


def block_sim(make, w, loader=True):
    """RotBond kn = ks = 1e5, kt = kb = 1e3, brittle strengths 0.5 / 1.0 / 1.0 / 0.5 (normal /
    shear / torsion / bending); RotFriction (same stiffness, mu 0.6) for post-failure contacts with
    the bond exclusion; elastic platens (k = 1e5) loading at a strain rate of 1e-4 per 1,000
    steps split between them; dt = 1e-5."""
    pos, rad = w["pos"], w["rad"]
    n = len(rad)
    s = make("RotSphere", 2.2, 0.2, (0, 0, 0), w["box"], (0, 0, 0), B_DT)
    s.add_particles(np.arange(n, dtype=np.int32), pos, rad, (4.0 / 3.0) * PI_REF * rad ** 3,
                    tag=np.zeros(n, np.int32))
    s.add_connections(np.ones(len(w["i1"]), np.int32), w["i1"], w["i2"])
    s.add_rot_bond_group("bonds", 1, 1e5, 1e5, 1e3, 1e3, 0.5, 1.0, 1.0, 0.5, True, True, 1.0)
    s.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, B_DT, True, True)
    s.add_exclusion("bonds", "friction")
    y0, y1 = float((pos[:, 1] - rad).min()), float((pos[:, 1] + rad).max())
    s.add_wall("bottom", (0, y0, 0), (0, 1, 0))
    s.add_wall("top", (0, y1, 0), (0, -1, 0))
    s.add_wall_group("bottom_w", "bottom", 1e5)
    s.add_wall_group("top_w", "top", 1e5)
    v = 0.5 * 1e-4 * (y1 - y0) / 1000 / B_DT
    if loader:  # the library's native wall loader (WallLoaderRunnable)
        s.set_wall_velocity("bottom", (0, v, 0))
        s.set_wall_velocity("top", (0, -v, 0))
    s.platen_step = v * B_DT  # per-step platen displacement, for a harness without a native loader
    return s


def bonded_block_leg(stream, steps=200, warm=20, cpu=True, cpu_budget=15.0, sweep_steps=10, n=1_000_000, tpp=0):
    """The 1M-sphere bonded block in both precision forms (device bond hand-off on), each on the
    step form (one lane, eight lanes or the tiled kernels) that measured fastest on a short run of
    the same block (or on `tpp` lanes when set), with the reference's own C++ (one core) on a
    bounded sample of the block."""
    from esys.lsm import _capi

    t0 = time.perf_counter()
    w = block_world(n)
    t_pack = time.perf_counter() - t0
    n = len(w["rad"])
    forms = {}
    for prec in (32, 64):
        sim = block_sim(lambda *a: _capi.DemSim(*a), w)
        sim.set_stream(stream.cuda_stream)
        sim.set_option("profile", 1)
        sim.set_option("precision", prec)
        sim.set_option("bond_handoff", 1)
        table = {}
        for t in ((tpp,) if tpp else (16, 8, 1)):
            sim.set_option("threads_per_particle", t)
            sim.step(2)
            table[t] = timed_run(sim, stream, sweep_steps)[0] / sweep_steps
        best = min(table, key=table.get)
        sim.set_option("threads_per_particle", best)
        sim.step(warm)
        ms, c0, c1 = timed_run(sim, stream, steps)
        cu = c1["contact_updates"] - c0["contact_updates"]
        kus = (c1["step_kernel_ns"] - c0["step_kernel_ns"]) / max(1, c1["profiled_steps"] - c0["profiled_steps"]) / 1e3
        nb = sim._chk(sim.lib.dem_num_pairs(sim.h, b"bonds"))
        mf = sim._chk(sim.lib.dem_num_pairs(sim.h, b"friction"))
        walls = c1["contacts_per_step"] - nb - mf
        st = sim.pairs("friction")[2]
        touching = int(st[:, 4].sum()) if len(st) else 0
        alg = n * 256 + nb * 32 + mf * (36 if prec == 32 else 60) + walls * 4
        forms[f"fp{prec}"] = {
            "value": cu / (ms / 1e3), "timesteps_per_s": steps / (ms / 1e3), "ms_per_timestep": ms / steps,
            "device_us_per_timestep": kus, "threads_per_particle": c1["threads_per_particle"],
            "intact_bonds": nb, "friction_pairs": mf, "touching_friction_pairs": touching, "wall_candidates": walls,
            "bond_breaks": int(len(sim.breaks()[0])),
            "lanes_sweep": {"chosen": best, "ms_per_timestep": {str(k): round(v, 4) for k, v in table.items()},
                            "timesteps_each": sweep_steps},
            "roofline": {"bound": "hbm", "achieved": alg / (kus * 1e-6) / 1e9, "unit": "GB/s",
                         "algorithmic_bytes_per_timestep": alg,
                         "kernels": "bond pass + step kernel per timestep (device time between CUDA events)"},
        }
        sim.close()
    peak, _ = peaks()
    for f in forms.values():
        f["roofline"]["frac"] = f["roofline"]["achieved"] / peak
    out = {
        "workload": f"bonded block: {n} RotSpheres fitted in {'x'.join(f'{b:g}' for b in w['box'])} (r in [0.2,1.0]), "
                    f"{len(w['i1'])} RotBonds "
                    f"(kn=ks=1e5, kt=kb=1e3, strengths 0.5/1.0/1.0/0.5), RotFriction + exclusion, platens at "
                    f"strain rate 1e-4 per 1,000 steps, dt=1e-5, device bond hand-off",
        "metric": "contact-updates/s", "timed_timesteps": steps, "warmup_timesteps": warm, "pack_s": t_pack,
        "forms": forms, "fp32_vs_fp64": forms["fp32"]["value"] / forms["fp64"]["value"], "cpu_reference": None,
    }
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        if oracle.available("ref"):
            t0 = time.perf_counter()
            r = block_sim(lambda *a: oracle.OracleSim("ref", *a), w, loader=False)
            t_set = time.perf_counter() - t0
            d = r.platen_step

            def load():  # the wall-loader runnable's moveWallBy ahead of each step
                r.move_wall("bottom", (0, d, 0))
                r.move_wall("top", (0, -d, 0))

            done, dt = cpu_sample(r, cpu_budget, 50, before=load)
            m_r = r.f["num_pairs"](r.h, b"friction") + r.f["num_pairs"](r.h, b"bonds")
            cand = forms["fp64"]["wall_candidates"]
            out["cpu_reference"] = {"value": (m_r + cand) * done / dt, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"{done} timesteps after set-up ({t_set:.0f} s) of the same block"}
            out["speedup_vs_cpu_reference"] = forms["fp32"]["value"] / out["cpu_reference"]["value"]
            del r
    return out


def window_bytes(n, m, nb, T, K):
    """Device bytes of one specimen's window: checkpoints every K of T steps (particle records,
    friction histories, wall candidacy) and the reverse pass's recompute of K + 1 states (records,
    FP32 velocity shadows and histories), pre-damping sums, damping counts and adjoints."""
    nseg = -(-T // K)
    return (n * (nseg * 132 + (K + 1) * 160 + K * 70 + 256) + m * (nseg * 32 + (K + 1) * 16 + 240)
            + nb * 170)


def ensemble_window_leg(sims, tpp, nsteps, every):
    """Batched differentiable window over the last ``nsteps`` steps of every specimen (FP32
    forces, FP64 integration and reverse): the window forward in batched chunks, then the
    reverse pass with one launch per kernel and step for all specimens of a batch.  Specimens
    are taken in batches that fit the free device memory.  Loss per specimen: MSE of its
    platen reactions vs a seeded ramp."""
    import torch

    from esys.lsm import _capi

    for s in sims:  # a fresh neighbour search: the whole verletDist/2 budget for the window
        s.search_neighbors()
    sizes = []
    for s in sims:
        n = s.num_particles()
        nb = len(s.pairs("bonds")[0])
        m = len(s.pairs("friction")[0]) + nb  # the friction list also holds the bond-excluded pairs
        sizes.append(window_bytes(n, m, nb, nsteps, every))
    budget = 0.6 * torch.cuda.mem_get_info()[0]
    batches, cur, used = [], [], 0
    for k, b in enumerate(sizes):
        if cur and used + b > budget:
            batches.append(cur)
            cur, used = [], 0
        cur.append(k)
        used += b
    if cur:
        batches.append(cur)
    t_fwd = t_rev = 0.0
    comps = 0
    loss = 0.0
    for grp in batches:
        e = _capi.Ensemble([sims[k] for k in grp])
        e.set_option("threads_per_particle", tpp)
        t0 = time.perf_counter()
        R = e.window_forward(nsteps, every)
        t1 = time.perf_counter()
        gR = []
        for r in R:
            tgt = window_target(r)
            loss += float(((r - tgt) ** 2).mean())
            gR.append(2.0 * (r - tgt) / r.size)
        G = e.window_adjoint(gR)
        t2 = time.perf_counter()
        t_fwd += t1 - t0
        t_rev += t2 - t1
        comps += sum(len(g["params"]) + g["vel"].size for g in G)
        e.close()
        for k in grp:
            sims[k].window_release()
    return {
        "workload": f"last {nsteps} steps of every specimen, checkpoints every {every}, "
                    f"{len(batches)} batch(es) by device memory",
        "loss": "per specimen: MSE of its platen reactions vs a seeded ramp",
        "dtype": "f32-forces/f64-integration forward and recompute, f64 reverse",
        "specimens": len(sims), "batches": len(batches), "window_bytes_estimate": int(sum(sizes)),
        "gradient_components": comps, "forward_with_checkpoints_s": t_fwd, "reverse_sweep_s": t_rev,
        "adjoint_grads_per_s": comps / (t_fwd + t_rev),
        # central differences: each batched forward window yields one perturbed loss per specimen
        "fd_grads_per_s": len(sims) / (2.0 * t_fwd),
        "adjoint_vs_fd_speedup": (comps / (t_fwd + t_rev)) / (len(sims) / (2.0 * t_fwd)),
        "loss_sum": loss,
    }


def ensemble_leg(nspec, steps, fp64_sample=32, fp64_steps=100, dist=None, window=200, window_every=20,
                 fp64_batched_steps=200):
    """FP32-force batched ensemble (autotuned, graph-replayed) vs the FP64 batched ensemble and
    the plain FP64 GPU form (each specimen stepped by itself), separating precision from batching.  Under torchrun each rank takes a size-balanced share of
    the specimens (no exchange while they run); counts are summed and times maxed at the end."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from esys.lsm import _capi
    from esys.lsm.autotune import autotune_ensemble
    from esys.lsm.parallel import partition_specimens, sharded_totals

    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    mine = partition_specimens([specimen_target_count(k) for k in range(nspec)], world)[rank]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(8) as ex:
        specs = list(ex.map(cylinder_specimen, mine))
    t_setup = time.perf_counter() - t0
    make = lambda *a: _capi.DemSim(*a)
    best, table = autotune_ensemble(lambda sp, g, sk: cylinder_sim(make, sp, g, sk), specs, 1.0,
                                    skins=(0.1, 0.2, 0.35), cell_factors=(1.0,), tpps=(2, 4, 8, 16), sample=24,
                                    warmup=30, trial=80)
    sims = [cylinder_sim(make, sp, best["grid_spacing"], best["verlet_dist"]) for sp in specs]
    for s in sims:
        s.set_option("precision", 32)
    e = _capi.Ensemble(sims)
    e.set_option("threads_per_particle", best["threads_per_particle"])
    e.set_option("profile", 1)
    e.step(100)  # warm-up: first searches, graph capture
    if dist is not None:
        torch.cuda.synchronize()
        dist.barrier()
    c0 = e.counters()
    t0 = time.perf_counter()
    e.step(steps)
    dt = time.perf_counter() - t0
    c1 = e.counters()
    contacts = float(c1["contact_updates"] - c0["contact_updates"])
    dt, contacts = sharded_totals(dt, contacts, dist, device="cuda")
    value = contacts / dt
    kern_ms = (c1["step_kernel_ns"] - c0["step_kernel_ns"]) / 1e6
    # FP32 force error vs FP64 on the developed states of a few specimens
    errs = []
    for s in sims[:: max(1, nspec // 8)]:
        s.set_option("precision", 64)
        errs.append(s.precision_report())
        s.set_option("precision", 32)
    breaks = int(sum(len(s.breaks()[0]) for s in sims))
    e.close()
    adj = None
    if window > 0:
        try:
            adj = ensemble_window_leg(sims, best["threads_per_particle"], window, window_every)
        except _capi.DemError as x:
            adj = {"failed": str(x)}
    for s in sims:
        s.close()
    # FP64 batched: the same specimens from their initial state, the ensemble in the FP64 form
    sims64 = [cylinder_sim(make, sp, best["grid_spacing"], best["verlet_dist"]) for sp in specs]
    for s in sims64:
        s.set_option("precision", 64)
    e64 = _capi.Ensemble(sims64)
    e64.set_option("threads_per_particle", best["threads_per_particle"])
    e64.step(100)  # warm-up as above
    if dist is not None:
        torch.cuda.synchronize()
        dist.barrier()
    b0 = e64.counters()
    t0 = time.perf_counter()
    e64.step(fp64_batched_steps)
    t_b64 = time.perf_counter() - t0
    c_b64 = float(e64.counters()["contact_updates"] - b0["contact_updates"])
    e64.close()
    for s in sims64:
        s.close()
    t_b64, c_b64 = sharded_totals(t_b64, c_b64, dist, device="cuda")
    batched64 = c_b64 / t_b64
    # plain FP64 GPU form: a size-stratified sample of the specimens, each stepped alone
    nloc = len(specs)
    idx = np.argsort([sp["n"] for sp in specs])[np.linspace(0, nloc - 1, min(max(1, fp64_sample // world), nloc)).astype(int)]
    c64 = 0
    t64 = 0.0
    for k in idx:
        s = cylinder_sim(make, specs[k], 2.2, 0.2)
        s.set_option("precision", 64)
        s.step(20)
        a = s.counters()
        t0 = time.perf_counter()
        s.step(fp64_steps)
        t64 += time.perf_counter() - t0
        c64 += s.counters()["contact_updates"] - a["contact_updates"]
        s.close()
    # every GPU runs its own sample: aggregate rate = sum of counts / max time
    t64, c64 = sharded_totals(t64, c64, dist, device="cuda")
    plain = c64 / t64
    return {
        "workload": f"{nspec} bonded cylinders (height 4R), particle counts log-uniform in [2,000, 40,000] "
                    f"({sum(sp['n'] for sp in specs)} on rank 0 of {world}), radii in [0.2, 1.0] by the fitting packer, "
                    f"kn, ks log-uniform [1e4, 1e6], strengths log-uniform [0.1, 2.0], RotFriction + exclusion, "
                    f"platens closing, dt=1e-5",
        "metric": "contact-updates/s", "value": value, "steps": steps, "seconds": dt,
        "batched_kernel_share": kern_ms / (dt * 1e3), "dtype": "f32-forces/f64-integration",
        "force_error_vs_fp64": {k: max(e[k] for e in errs) for k in errs[0]} if errs else None,
        "force_error_sample": f"{len(errs)} specimens, FP32 forces vs FP64 on their developed states",
        "bond_breaks": breaks,
        "autotuned": best, "autotune_trials": len(table), "setup_s": t_setup,
        "plain_fp64_gpu": {"value": plain, "sample": f"{len(idx)} specimens per GPU (size-stratified) x "
                                                      f"{fp64_steps} steps each, one dem_step per specimen"},
        "scaling": "weak over specimens: each GPU advances its size-balanced share, no exchange" if world > 1
                   else "single GPU",
        "fp64_batched": {"value": batched64, "steps": fp64_batched_steps,
                         "sample": "the same specimens from their initial state, batched in the FP64 form"},
        "speedup_vs_plain_fp64": value / plain,
        "fp32_batched_vs_fp64_batched": value / batched64,
        "fp64_batched_vs_plain_fp64": batched64 / plain,
        "batched_adjoint": adj,
    }


def run_reference_arm(args):
    """The reference's own C++ (oracle/_ref: ESyS-Particle's hot-path classes compiled from its
    sources, one worker = one core) on the headline packing, through the same steps and
    warm-up counts as the GPU arm; one "step" here is one timestep (a bounded sample of the
    GPU arm's --dem-steps).  The packing comes from the packer linked into the reference
    library, so this arm maps no product library.  Periodic x needs >= 2 MPI workers in the
    reference, so it runs the same particles and groups in a non-periodic box."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.available("ref"):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
        return
    w = workload(packer=oracle.rsi_pack_ref)
    sim = setup(lambda *a: oracle.OracleSim("ref", *a), w, periodic=False)
    sim.step(1)  # first step: neighbour search + interaction set-up (not timed)
    m = sim.f["num_pairs"](sim.h, b"friction")
    pos = w["pos"]
    ncand = int((np.abs(pos[:, 1] - 0.0) < GRID).sum() + (np.abs(pos[:, 1] - 50.0) < GRID).sum())
    for _ in range(args.warmup):
        sim.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(1)
    dt = time.perf_counter() - t0
    value = (m + ncand) * args.steps / dt
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded RSI packing)",
        "impl": "reference",
        "config": {"workload": HEADLINE_WORKLOAD, "particles": len(w["ids"]),
                   "periodic_x": False,
                   "reference_note": "the reference needs >= 2 MPI workers for periodic x; one worker runs the "
                                     "same particles and groups non-periodic",
                   "timesteps_per_step": 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} timesteps after {args.warmup} warm-up timesteps of the "
                                   f"250k-sphere packing, {m} friction pairs + {ncand} wall candidates"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--dem-steps", type=int, default=200, help="timesteps per bench step")
    ap.add_argument("--tpp", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64],
                    help="32: FP32 pair forces + FP64 integration (headline); 64: FP64 throughout")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-window leg")
    ap.add_argument("--no-widened", action="store_true", help="skip the NRotFriction leg")
    ap.add_argument("--ensemble-specimens", type=int, default=512, help="0 skips the batched-ensemble leg")
    ap.add_argument("--ensemble-steps", type=int, default=1000, help="timed timesteps of the ensemble leg")
    ap.add_argument("--ensemble-window", type=int, default=200,
                    help="steps of the batched differentiable window after the ensemble run (0 skips)")
    ap.add_argument("--ensemble-window-every", type=int, default=20, help="checkpoint interval of that window")
    ap.add_argument("--split", type=int, default=-1, choices=[-1, 0, 1],
                    help="step kernels: -1 automatic, 0 fused, 1 pair kernel + integration kernel")
    ap.add_argument("--no-gravity", action="store_true", help="skip the 8,000-sphere gravity-packing leg")
    ap.add_argument("--no-block", action="store_true", help="skip the 1M-sphere bonded-block leg")
    ap.add_argument("--block-steps", type=int, default=200, help="timed timesteps of the bonded-block leg")
    ap.add_argument("--block-particles", type=int, default=1_000_000, help="spheres of the bonded block")
    ap.add_argument("--block-tpp", type=int, default=0, help="lanes per particle of the bonded block (0: measured)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from esys.lsm import _capi

    w = workload()
    n = len(w["ids"])
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def make_sim(precision):
        sim = setup(lambda *a: _capi.DemSim(*a), w, periodic=True)
        sim.set_stream(stream.cuda_stream)
        sim.set_option("profile", 1)
        sim.set_option("precision", precision)
        sim.set_option("split", args.split)
        if args.tpp:
            sim.set_option("threads_per_particle", args.tpp)
        sim.set_wall_velocity("bottom", (-0.01, 0, 0))
        sim.set_wall_velocity("top", (0.01, 0, 0))
        return sim

    def bench_step(sim):
        sim.step(args.dem_steps)
        sim.apply_force_to_wall("top_w", (0.0, -NORMAL_LOAD, 0.0))

    sweeps = {}

    def pick_lanes(sim, label):
        """Lanes per particle measured on this workload before the timed steps: one lane, two
        lanes, and the warp-cooperative pair sums (32); the fastest is kept."""
        if args.tpp:
            return
        table = {}
        for t in (1, 2, 32):
            sim.set_option("threads_per_particle", t)
            bench_step(sim)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(2):
                bench_step(sim)
            e1.record(stream)
            torch.cuda.synchronize()
            table[t] = e0.elapsed_time(e1) / 2
        best = min(table, key=table.get)
        sim.set_option("threads_per_particle", best)
        sweeps[label] = {"chosen": best, "ms_per_bench_step": {str(k): round(v, 4) for k, v in table.items()}}

    def timed(sim, clk=None):
        for _ in range(args.warmup):
            bench_step(sim)
            flush.zero_()
        barrier()
        c0 = sim.counters()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            bench_step(sim)
            ev[k][1].record(stream)
        barrier()
        c1 = sim.counters()
        return c0, c1, sum(a.elapsed_time(b) for a, b in ev)

    fp64 = None
    if args.precision == 32 and not args.no_fp64_compare:
        s64 = make_sim(64)
        pick_lanes(s64, "fp64")
        a0, a1, ms64 = timed(s64)
        ns64 = (a1["step_kernel_ns"] - a0["step_kernel_ns"]) / max(1, a1["profiled_steps"] - a0["profiled_steps"])
        fp64 = {"value": (a1["contact_updates"] - a0["contact_updates"]) / (ms64 / 1e3), "kernel_us": ns64 / 1e3,
                "ms_per_step": ms64 / args.steps}
        s64.close()
    sim = make_sim(args.precision)
    pick_lanes(sim, "fp32" if args.precision == 32 else "fp64")
    with Clocks(local) as clk:
        c0, c1, ms = timed(sim)
    err = None
    if args.precision == 32:
        # force error of the FP32 form vs FP64 on the developed state (same positions, velocities, history)
        sim.set_option("precision", 64)
        err = sim.precision_report()
        sim.set_option("precision", 32)
    contacts = c1["contact_updates"] - c0["contact_updates"]
    fst = sim.pairs("friction")[2]
    touching = int(fst[:, 4].sum()) if len(fst) else 0  # touching RotFriction pairs after the timed steps
    t_max = ms
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        cc = torch.tensor([float(contacts)], device="cuda", dtype=torch.float64)
        dist.all_reduce(cc)
        contacts_all = float(cc.item())
    else:
        contacts_all = float(contacts)
    value = contacts_all / (t_max / 1e3)

    # dominant kernel: the force + integration kernel, timed with CUDA events on its stream
    step_ns = (c1["step_kernel_ns"] - c0["step_kernel_ns"]) / max(1, c1["profiled_steps"] - c0["profiled_steps"])
    m_fric = sim._chk(sim.lib.dem_num_pairs(sim.h, b"friction"))
    n_wall_cand = c1["contacts_per_step"] - m_fric
    # algorithmic bytes per launch: particle 256 B (rot, FP64), RotFriction pair 60 B (FP32 history: 36 B),
    # wall candidate 4 B
    alg_bytes = n * 256 + m_fric * (36 if args.precision == 32 else 60) + n_wall_cand * 4
    achieved = alg_bytes / (step_ns * 1e-9) / 1e9
    peak, peak_kind = peaks()
    tpp_used = c1["threads_per_particle"]
    kernel_name = (f"k_step<ROT=1, TPP={tpp_used}, FRIC, {'FP32' if args.precision == 32 else 'FP64'}>"
                   if tpp_used != 16 else f"k_step_tiled<ROT=1, FRIC, {'FP32' if args.precision == 32 else 'FP64'}>")
    traffic = traffic_per_launch()
    # the ncu capture's traffic counts only for the same kernel instance
    traffic_bytes = traffic["bytes_per_launch"] if traffic and traffic.get("kernel", "").startswith(kernel_name) else None

    # e2e through the C ABI with host buffers (pinned), H2D + D2H inside the timed region
    pin = {k: torch.empty((n, wdt), dtype=torch.float64).pin_memory() for k, wdt in
           (("pos", 3), ("vel", 3), ("angvel", 3), ("quat", 4), ("force", 3), ("moment", 3))}
    ids_pin = torch.empty(n, dtype=torch.int32).pin_memory()
    sim.get_particles_raw(ids_pin.data_ptr(), *(pin[k].data_ptr() for k in ("pos", "vel", "angvel", "quat", "force",
                                                                             "moment")))
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    ce0 = sim.counters()
    e2e_sec = 0.0
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        s0 = time.perf_counter()
        sim.set_particles(pos=pin["pos"].data_ptr(), vel=pin["vel"].data_ptr(), angvel=pin["angvel"].data_ptr(),
                          quat=pin["quat"].data_ptr(), n=n)
        bench_step(sim)
        sim.get_particles_raw(ids_pin.data_ptr(), *(pin[k].data_ptr() for k in ("pos", "vel", "angvel", "quat",
                                                                                 "force", "moment")))
        s1 = time.perf_counter()
        e2e_sec += s1 - s0
    ce1 = sim.counters()
    e2e_contacts = ce1["contact_updates"] - ce0["contact_updates"]
    e2e_val = e2e_contacts / e2e_sec
    if dist is not None:
        t = torch.tensor([e2e_sec], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        cc = torch.tensor([float(e2e_contacts)], device="cuda", dtype=torch.float64)
        dist.all_reduce(cc)
        e2e_val = float(cc.item()) / float(t.item())

    adj = None
    if not args.no_adjoint:
        adj = adjoint_leg(stream)
    nrot = None
    if not args.no_widened and world == 1:
        nrot = nrot_friction_leg(stream)
    grav = None
    if not args.no_gravity and world == 1:
        grav = gravity_leg(stream, cpu=not args.no_cpu_baseline)
    block = None
    if not args.no_block and world == 1:
        block = bonded_block_leg(stream, steps=args.block_steps, cpu=not args.no_cpu_baseline, n=args.block_particles,
                                 tpp=args.block_tpp)
    ens = None
    if args.ensemble_specimens > 0:
        ens = ensemble_leg(args.ensemble_specimens, args.ensemble_steps, dist=dist, window=args.ensemble_window,
                           window_every=args.ensemble_window_every)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = cpu_reference_sample(w, steps=30, timeout_s=25.0)
        if res is not None:
            cpu = {"value": res["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"{res['steps']} timesteps of the same 250k-sphere packing (non-periodic: the reference "
                             f"needs >=2 MPI workers for periodic x), after set-up; {res['pairs']} friction pairs"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-forces/f64-integration" if args.precision == 32 else "f64",
            "data": "synthetic (seeded RSI packing)",
            "config": {"workload": HEADLINE_WORKLOAD, "periodic_x": True,
                       "dem_steps_per_step": args.dem_steps, "particles": n,
                       "interactions_per_timestep": c1["contacts_per_step"],
                       "friction_pairs": m_fric, "wall_candidates": n_wall_cand,
                       "touching_friction_pairs": touching,
                       "threads_per_particle": c1["threads_per_particle"],
                       "lanes_sweep": sweeps,
                       "l2": "flushed (256 MB write) between bench steps; the step's working set (~110 MB) is "
                             "close to the 126 MB L2, so part of it stays resident between timesteps",
                       "parallelism": "replicas only" if world > 1 else "single GPU",
                       "precision": ("FP32 pair forces (Kahan-compensated), FP64 positions / contact detection / "
                                     "integration" if args.precision == 32 else "FP64 throughout"),
                       "force_error_vs_fp64": err if err is not None else {"max_rel_force_err": 0.0},
                       "fp64_form": fp64},
            "timesteps_per_s": args.dem_steps * args.steps / (t_max / 1e3),
            "touching_contact_updates_per_s": value * touching / max(1, c1["contacts_per_step"]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic_bytes, "traffic_kernel": (traffic or {}).get("kernel"),
                         "kernel": kernel_name, "kernel_us": step_ns / 1e3,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": n * (24 + 24 + 24 + 32),
                    "d2h_bytes_per_step": n * (4 + 5 * 24 + 32)},
            "gpu_launches": c1["launches"] - c0["launches"],
            "clocks": clk.summary(),
            "adjoint": adj,
            "nrot_friction": nrot,
            "ensemble": ens,
            "gravity_packing": grav,
            "bonded_block": block,
        }
        print(json.dumps(line, default=_jsonable))
    sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
