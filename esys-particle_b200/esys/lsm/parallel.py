"""Specimen-parallel ensembles over several GPUs (one process per GPU).

Independent specimens need no exchange while they run: each rank advances its
own share as one batched ensemble, and results meet once at the end (a gather of
per-specimen results, and sums / maxima of the throughput counters).  Shares are
balanced by particle count with the longest-processing-time rule: specimens in
decreasing size, each to the rank with the least work so far (ties to the lower
rank), which keeps the largest share within one specimen of the mean.
"""
from __future__ import annotations

import numpy as np

__all__ = ["partition_specimens", "gather_objects"]


def partition_specimens(sizes, world):
    """Indices of the specimens of each rank (each list ascending), balanced by size."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world, dtype=np.int64)
    parts = [[] for _ in range(world)]
    for k in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        parts[r].append(int(k))
        load[r] += sizes[k]
    return [sorted(p) for p in parts]


def gather_objects(obj, dist=None):
    """All ranks' objects in rank order (one collective); [obj] without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
