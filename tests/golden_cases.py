"""Golden-fixture cases: small seeded scenarios whose outputs, produced by the
reference's own code (oracle/_ref), are committed under tests/golden/ by
tests/golden/make_golden.py.  The same runner drives the CPU restatement and
the CUDA path in the tests."""
from __future__ import annotations

import numpy as np

import scenarios as S

CASES = {
    # name: (builder, groups, walls, driver)
    "gravity_box": (lambda mk: S.gravity_box(mk, 5), ["elastic"], ["xlo", "zlo", "zhi"], ("steps", 120)),
    "friction_pack": (lambda mk: S.friction_pack(mk), ["friction"], ["floor", "roof"], ("steps", 120)),
    "bonded_block": (lambda mk: S.bonded_block(mk, strength=(0.05, 0.1, 0.1, 0.05)), ["bonds", "friction"],
                     ["bottom", "top"], ("loaded", 200, 2e-4)),
}


def run(name, mk):
    build, groups, walls, drv = CASES[name]
    sim = build(mk)
    if drv[0] == "steps":
        sim.step(drv[1])
    else:
        S.run_loaded(sim, drv[1], drv[2])
    return sim


def collect(name, sim):
    _, groups, walls, _ = CASES[name]
    p = sim.particles()
    out = {k: p[k] for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment")}
    for g in groups:
        a, b, st = sim.pairs(g)
        out[f"pairs_{g}_id1"], out[f"pairs_{g}_id2"], out[f"pairs_{g}_state"] = a, b, st
    for w in walls:
        pos, f = sim.wall(w)
        out[f"wall_{w}_pos"], out[f"wall_{w}_force"] = pos, f
    if "bonds" in groups:
        a, b, s = sim.breaks()
        out["breaks_id1"], out["breaks_id2"], out["breaks_step"] = a, b, s
    return out


def assert_matches(g, sim, exact, name, rtol_pos=1e-9, rtol_force=1e-8):
    """exact: bit-identical (CPU restatement).  Otherwise: identical pair/event
    sets and fields within the stated tolerances relative to each field's scale."""
    got = collect(name, sim)
    for k in g.files:
        a, b = g[k], got[k]
        assert a.shape == b.shape, (k, a.shape, b.shape)
        if exact or k.endswith(("id1", "id2", "_step")) or k == "id":
            assert np.array_equal(a, b), k
            continue
        if k.endswith("_state"):
            # Only RotFriction keeps per-pair state on the CUDA path (tangential force,
            # slipping, touching); elastic pairs are stateless and bonds keep no record.
            if a.size and "friction" in k:
                assert np.array_equal(a[:, 3:], b[:, 3:]), k
                scale = max(np.abs(a[:, :3]).max(), 1e-300)
                assert np.abs(a[:, :3] - b[:, :3]).max() <= rtol_force * scale, k
            continue
        scale = max(np.abs(a).max(), 1e-300)
        tol = rtol_force if ("force" in k or "moment" in k) else rtol_pos
        assert np.abs(a - b).max() <= tol * scale, (k, np.abs(a - b).max(), scale)
