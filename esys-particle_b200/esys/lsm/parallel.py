"""Specimen-parallel ensembles over several GPUs (one process per GPU).

Independent specimens need no exchange while they run: each rank advances its
own share as one batched ensemble, and results meet once at the end (a gather of
per-specimen results, and sums / maxima of the throughput counters).  Shares are
balanced by a per-specimen work figure with the longest-processing-time rule:
specimens in decreasing work, each to the rank with the least work so far (ties
to the lower rank), which keeps the largest share within one specimen of the
mean.  The work of a specimen is its particle count times its interactions per
particle, N_s * (M / N); for specimens cut from one packer the interactions per
particle are nearly equal, and the particle count alone stands for it.

The helpers take the process group (or None for one process) and do not care
what steps a specimen: the bench's ranks run the CUDA ensemble, the CPU tests'
ranks run the oracle, through the same calls.
"""
from __future__ import annotations

import numpy as np

__all__ = ["partition_specimens", "gather_objects", "sharded_totals", "run_share"]


def partition_specimens(sizes, world, per_particle=None):
    """Indices of the specimens of each rank (each list ascending), balanced by work: sizes[k],
    times per_particle[k] (interactions per particle) when given."""
    sizes = np.asarray(sizes, dtype=np.float64 if per_particle is not None else np.int64)
    if per_particle is not None:
        sizes = sizes * np.asarray(per_particle, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world, dtype=sizes.dtype)
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


def sharded_totals(seconds, count, dist=None, device="cpu"):
    """A sharded run's time and work: the slowest rank's seconds and the sum of every rank's
    count (two all-reduces, taken by every rank in the same order).  `device` holds the
    reduction tensors: "cuda" under NCCL, "cpu" under gloo."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds), float(count)
    import torch

    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def run_share(sizes, build, run, dist=None, per_particle=None):
    """This rank's part of an ensemble: its balanced share of the specimens, each built by
    build(k), all advanced together by run(specimens) -> {k: result}, then every rank's results
    merged by one gather.  Returns (merged results of all specimens, this rank's indices)."""
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    mine = partition_specimens(sizes, world, per_particle)[rank]
    results = run({k: build(k) for k in mine})
    merged = {}
    for part in gather_objects(results, dist):
        merged.update(part)
    return merged, mine
