"""Slab decomposition (esys.lsm.slabs) with the GPU library's handles as the slab workers, all on
one device in one process (the exchange goes through host arrays; one process per GPU uses the
same worker code over a process group, see tests/test_slabs.py), against the same specimen on one
handle.  Bar as in tests/test_slabs.py."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


def _compare(dom, single, rtol_pos=1e-12, rtol_f=1e-10):
    pa, pb = dom.particles(), single.particles()
    assert np.array_equal(pa["id"], pb["id"]), (len(pa["id"]), len(pb["id"]))
    for k, tol in (("pos", rtol_pos), ("vel", rtol_pos), ("force", rtol_f)):
        scale = max(np.abs(pb[k]).max(), 1e-300)
        assert np.abs(pa[k] - pb[k]).max() <= tol * scale, k
    x, y = dom.pairs("friction", touching_only=True), single.pairs("friction")
    t = y[2][:, 4] > 0
    assert np.array_equal(x[0], y[0][t]) and np.array_equal(x[1], y[1][t])


def test_gpu_slabs_with_migration_match_one_handle(gpu):
    edit = S.drift_x(20.0)
    dom = S.split(gpu, 3, S.wide_friction_pack, edit=edit)
    single = S.replay(gpu, S.wide_friction_pack, edit=edit)
    owned0 = [set(w.owned) for w in dom.workers]
    for _ in range(10):
        dom.step(200)
        single.step(200)
        _compare(dom, single)
    assert dom.repartitions > 20
    assert sum(len(o - set(w.owned)) for o, w in zip(owned0, dom.workers)) > 30
    dom.close()


def test_gpu_slabs_bonded_block_failures_match_one_handle(gpu):
    kw = dict(strength=(0.4, 0.8, 0.8, 0.4))
    dom = S.split(gpu, 2, S.bonded_block, **kw)
    single = S.replay(gpu, S.bonded_block, **kw)
    S.run_loaded(dom, 150, 0.002)
    S.run_loaded(single, 150, 0.002)
    eb = sorted(zip(*(x.tolist() for x in single.breaks())), key=lambda e: (e[2], e[0], e[1]))
    assert len(eb) > 0 and dom.breaks() == eb
    _compare(dom, single)
    for w in ("top", "bottom"):
        fa, fb = dom.wall(w)[1], single.wall(w)[1]
        assert np.abs(fa - fb).max() <= 1e-10 * max(np.abs(fb).max(), 1.0), w
    dom.close()
