"""Specimen-parallel ensembles: the partition and the end-of-run gather, on CPU ranks
(gloo, world size 2), as the multi-GPU bench runs them with one rank per GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from esys.lsm.parallel import gather_objects, partition_specimens


def test_partition_covers_each_specimen_once_and_balances():
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(40000), size=512)).astype(int)
    for world in (1, 2, 3, 8):
        parts = partition_specimens(sizes, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, sizes, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition_specimens(sizes, world)[rank]
    # each rank "runs" its share; the results meet once at the end
    res = {k: int(sizes[k]) * 3 for k in mine}
    allres = gather_objects(res, dist)
    if rank == 0:
        merged = {}
        for r in allres:
            merged.update(r)
        q.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_share_and_gather():
    sizes = np.array([40000, 2000, 15000, 9000, 7000, 30000, 2500])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert merged == {k: int(v) * 3 for k, v in enumerate(sizes)}
