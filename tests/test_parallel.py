"""Specimen-parallel ensembles: the partition and the end-of-run gather, on CPU ranks
(gloo, world size 2), as the multi-GPU bench runs them with one rank per GPU.  The
helpers of esys.lsm.parallel do not care what steps a specimen; here the ranks step
small bonded blocks with the oracle, where the bench's ranks run the CUDA ensemble."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from esys.lsm.parallel import gather_objects, partition_specimens, run_share, sharded_totals


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


def test_partition_by_work_per_particle():
    """N_s * (M / N): a small specimen with many interactions per particle weighs like a large one."""
    parts = partition_specimens([1000, 1000, 500], 2, per_particle=[1.0, 1.0, 4.0])
    assert sorted(map(sorted, parts)) == [[0, 1], [2]]


def test_partition_edges():
    """More ranks than specimens leaves the extra ranks empty; no specimens gives empty shares;
    a world below one is refused; without a process group the helpers act on the one process."""
    assert partition_specimens([7, 3], 4) == [[0], [1], [], []]
    assert partition_specimens([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition_specimens([1], 0)
    merged, mine = run_share([4, 2], lambda k: 10 * k, lambda sims: {k: v + 1 for k, v in sims.items()})
    assert merged == {0: 1, 1: 11} and mine == [0, 1]
    assert sharded_totals(2.5, 7) == (2.5, 7.0)


# Specimen k of the stepped test: a small bonded block (seed and height from k) under platen loading.
_SPEC_STEPS = 40


def _spec_sizes():
    return np.array([5 * (5 + k) * 5 for k in range(5)])


def _build_spec(k):
    import oracle
    import scenarios as S

    make = lambda *a: oracle.OracleSim("orc", *a)
    return S.bonded_block(make, nx=5, ny=5 + k, nz=5, seed=20 + k, strength=(0.2 + 0.1 * k, 0.5, 0.5, 0.3))


def _run_specs(sims):
    import scenarios as S

    out = {}
    for k, s in sims.items():
        S.run_loaded(s, _SPEC_STEPS, 0.002)
        p = s.particles()
        out[k] = {"pos": p["pos"], "breaks": len(s.breaks()[0]), "top": s.wall("top")[1]}
    return out


def _stepping_rank(rank, world, port, q):
    import time

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t0 = time.perf_counter()
    merged, mine = run_share(_spec_sizes(), _build_spec, _run_specs, dist)
    secs, count = sharded_totals(time.perf_counter() - t0, len(mine), dist)
    if rank == 0:
        q.put((merged, secs, count))
    dist.barrier()
    dist.destroy_process_group()


def _result(q, procs, limit):
    """The queue's item; stops the ranks and fails at once when one of them exits with an error."""
    import queue
    import time

    deadline = time.monotonic() + limit
    while True:
        try:
            return q.get(timeout=2)
        except queue.Empty:
            failed = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            if failed or time.monotonic() > deadline:
                for p in procs:
                    if p.is_alive():
                        p.kill()
                raise AssertionError(f"a rank failed (exit codes {failed})" if failed else "ranks timed out")


def test_two_ranks_step_their_shares():
    """Each gloo rank builds and steps only its share; the gathered per-specimen results equal one
    process stepping every specimen, and the totals count every specimen once."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_stepping_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, secs, count = _result(q, procs, 300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    alone, mine = run_share(_spec_sizes(), _build_spec, _run_specs)
    assert mine == list(range(5)) and count == 5 and secs > 0
    assert sorted(merged) == list(range(5))
    for k in range(5):
        assert np.array_equal(merged[k]["pos"], alone[k]["pos"]), k
        assert merged[k]["breaks"] == alone[k]["breaks"]
        assert np.array_equal(merged[k]["top"], alone[k]["top"])
    assert sum(alone[k]["breaks"] for k in range(5)) > 0
