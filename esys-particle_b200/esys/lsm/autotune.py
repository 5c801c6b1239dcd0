"""Autotuner of the batched ensemble: cell size, Verlet skin and threads per particle.

The three knobs trade against each other: a larger skin rebuilds less often but
carries more non-touching pairs through every step; a larger cell (grid spacing,
at least 2 r_max + skin) makes fewer, longer cell lists for the rebuild; more
threads per particle shorten each particle's adjacency walk at the cost of idle
lanes on short lists.  The tuner builds a size-stratified sample of the
specimens for every (cell, skin) candidate, runs a short trial of every
threads-per-particle setting through the ensemble, and keeps the fastest by
measured contact-updates per second (warm-up steps excluded).

Skin and cell size are the reference's ``verletDist`` and ``gridSpacing``: like
there, they decide when the neighbour lists are rebuilt, which for RotFriction
decides when separated pairs lose their history, so the tuned values are
recorded with every result.
"""
from __future__ import annotations

import time

import numpy as np

from . import _capi

__all__ = ["autotune_ensemble"]


def _sample(specs, k):
    if len(specs) <= k:
        return list(specs)
    sizes = np.array([s["n"] for s in specs])
    order = np.argsort(sizes, kind="stable")
    pick = order[np.linspace(0, len(specs) - 1, k).round().astype(int)]
    return [specs[i] for i in pick]


def autotune_ensemble(build, specs, r_max, skins=(0.1, 0.2, 0.35), cell_factors=(1.0, 1.3), tpps=(1, 2, 4, 8),
                      sample=32, warmup=40, trial=120, precision=32):
    """build(spec, grid_spacing, verlet_dist) -> DemSim.  Each spec is a dict with its particle
    count under "n".  Returns (best, table): best = dict(grid_spacing, verlet_dist,
    threads_per_particle, contact_updates_per_s); table lists every trial."""
    chosen = _sample(specs, sample)
    table = []
    for skin in skins:
        for f in cell_factors:
            cell = f * (2.0 * r_max + skin)
            sims = [build(s, cell, skin) for s in chosen]
            for s in sims:
                s.set_option("precision", precision)
            e = _capi.Ensemble(sims)
            e.set_option("chunk", 40)
            for tpp in tpps:
                e.set_option("threads_per_particle", tpp)
                e.step(warmup)
                c0 = e.counters()
                t0 = time.perf_counter()
                e.step(trial)
                dt = time.perf_counter() - t0
                c1 = e.counters()
                table.append({"grid_spacing": cell, "verlet_dist": skin, "threads_per_particle": tpp,
                              "contact_updates_per_s": (c1["contact_updates"] - c0["contact_updates"]) / dt})
            e.close()
            for s in sims:
                s.close()
    best = max(table, key=lambda r: r["contact_updates_per_s"])
    return dict(best), table
