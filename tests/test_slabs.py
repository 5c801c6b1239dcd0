"""Slab decomposition of one specimen (esys.lsm.slabs) on CPU workers: the CPU restatement as the
worker engine, in one process and as two gloo ranks, against the same specimen on one worker.

Bar: touching pair sets and bond-failure events exact; positions within 1e-12 and forces within
1e-10 of each field's scale (the slabs sum a particle's contributions in another order)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import scenarios as S
from esys.lsm.slabs import SlabLayout


@pytest.fixture(scope="module")
def orc(oracle_libs):
    return lambda *a: oracle_libs.OracleSim("orc", *a)


def _compare(dom, single, rtol_pos=1e-12, rtol_f=1e-10, group="friction"):
    pa, pb = dom.particles(), single.particles()
    assert np.array_equal(pa["id"], pb["id"]), (len(pa["id"]), len(pb["id"]))
    for k, tol in (("pos", rtol_pos), ("vel", rtol_pos), ("force", rtol_f)):
        scale = max(np.abs(pb[k]).max(), 1e-300)
        assert np.abs(pa[k] - pb[k]).max() <= tol * scale, k
    x, y = dom.pairs(group, touching_only=True), single.pairs(group)
    t = y[2][:, 4] > 0
    assert np.array_equal(x[0], y[0][t]) and np.array_equal(x[1], y[1][t])


def test_layout_is_cell_aligned_and_covers_the_box():
    L = SlabLayout((0, 0, 0), (10.0, 4.0, 3.0), 1.2, 3)
    assert L.axis == 0
    assert np.allclose(L.edges[:-1] / 1.2, np.round(L.edges[:-1] / 1.2))
    assert L.edges[0] == 0 and L.edges[-1] == 10.0
    assert list(L.owner([0.0, 4.7, 9.99, 12.0])) == [0, 1, 2, 2]
    with pytest.raises(ValueError):
        SlabLayout((0, 0, 0), (10.0, 4.0, 3.0), 1.2, 3, circ=(1, 0, 0), axis=0)


def test_split_friction_pack_with_migration_matches_one_worker(orc):
    """A frictional pack drifting along the split axis over three slabs: particles change slab
    (with the histories of their pairs) many times, and the trajectory stays the one-worker one."""
    edit = S.drift_x(20.0)
    dom = S.split(orc, 3, S.wide_friction_pack, edit=edit)
    single = S.replay(orc, S.wide_friction_pack, edit=edit)
    owned0 = [set(w.owned) for w in dom.workers]
    for _ in range(10):
        dom.step(200)
        single.step(200)
        _compare(dom, single)
    assert dom.repartitions > 20
    assert sum(len(o - set(w.owned)) for o, w in zip(owned0, dom.workers)) > 30  # particles migrated


def test_split_bonded_block_failures_match_one_worker(orc):
    """A loaded bonded block split across its loading axis: bond failures (events exact), the
    bond-to-friction hand-off and the platen reactions summed over slabs."""
    kw = dict(strength=(0.4, 0.8, 0.8, 0.4))
    dom = S.split(orc, 2, S.bonded_block, **kw)
    single = S.replay(orc, S.bonded_block, **kw)
    S.run_loaded(dom, 150, 0.002)
    S.run_loaded(single, 150, 0.002)
    eb = sorted(zip(*(x.tolist() for x in single.breaks())), key=lambda e: (e[2], e[0], e[1]))
    assert len(eb) > 0 and dom.breaks() == eb
    _compare(dom, single)
    for w in ("top", "bottom"):
        fa, fb = dom.wall(w)[1], single.wall(w)[1]
        assert np.abs(fa - fb).max() <= 1e-10 * max(np.abs(fb).max(), 1.0), w


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "esys-particle_b200"), os.path.join(root, "oracle"), here):
        if p not in sys.path:
            sys.path.insert(0, p)
    import oracle
    import scenarios as S2
    from esys.lsm.slabs import TorchTransport

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    orc = lambda *a: oracle.OracleSim("orc", *a)
    dom = S2.split(orc, world, S2.wide_friction_pack, edit=S2.drift_x(20.0), transport=TorchTransport(dist))
    dom.step(1200)
    parts = dom.particles()
    pairs = dom.pairs("friction", touching_only=True)
    if rank == 0:
        q.put((parts, pairs[:2], dom.repartitions))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_one_worker(orc):
    """One slab per process, exchanging over a gloo process group (the transport GPU ranks use
    with NCCL), against the one-worker run."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, pairs, nrep = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    single = S.replay(orc, S.wide_friction_pack, edit=S.drift_x(20.0))
    single.step(1200)
    pb = single.particles()
    assert np.array_equal(parts["id"], pb["id"])
    assert np.abs(parts["pos"] - pb["pos"]).max() <= 1e-12 * np.abs(pb["pos"]).max()
    y = single.pairs("friction")
    t = y[2][:, 4] > 0
    assert np.array_equal(pairs[0], y[0][t]) and np.array_equal(pairs[1], y[1][t])
    assert nrep > 5
