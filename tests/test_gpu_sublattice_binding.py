"""A master drives TGpuSubLattice (esys-particle_b200/integration/GpuSubLattice.h) through the
reference's command and buffer protocol (tests/binding: CLatticeMaster's sends, the worker's
command loop, the reference's own buffers and particle packing), and the specimen it builds
steps as the library driven directly does and as the CPU oracle does.  All tests need a GPU.

Bar: against the library driven directly 1e-12 of each field's largest magnitude (the master's
neighbour-search orders may move a rebuild, which reorders sums); against the oracle the parity
bar of the GPU parity tests (positions 1e-9, forces 1e-8 after hundreds of steps)."""
import numpy as np
import pytest

import binding_driver as B
import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def makers(binding_lib, oracle_libs):
    from esys.lsm import _capi

    return {
        "binding": lambda *a: B.SubLatticeMaster(binding_lib, *a),
        "direct": lambda *a: _capi.DemSim(*a),
        "oracle": lambda *a: oracle_libs.OracleSim("orc", *a),
    }


def _compare(a, b, tol_pos, tol_f, rot):
    pa, pb = a.particles(), b.particles()
    assert np.array_equal(pa["id"], pb["id"])
    keys = [("pos", tol_pos), ("vel", tol_pos), ("force", tol_f)]
    if rot:
        keys += [("angvel", tol_pos), ("quat", tol_pos), ("moment", tol_f)]
    for k, tol in keys:
        scale = max(np.abs(pb[k]).max(), 1e-300)
        err = np.abs(pa[k] - pb[k]).max()
        assert err <= tol * scale, (k, err, scale)


def test_bonded_block_through_the_binding(makers):
    sims = {k: S.bonded_block(m, strength=(0.05, 0.1, 0.1, 0.05)) for k, m in makers.items()}
    try:
        for s in sims.values():
            S.run_loaded(s, 300, 2e-4)
        a, d, o = sims["binding"], sims["direct"], sims["oracle"]
        assert a.num_particles() == d.num_particles() == len(o.particles()["id"])
        _compare(a, d, 1e-12, 1e-12, True)
        _compare(a, o, 1e-9, 1e-8, True)
        for w in ("top", "bottom"):
            pa, fa = a.wall(w)
            pd, fd = d.wall(w)
            po, fo = o.wall(w)
            assert np.array_equal(pa, pd) and np.abs(pa - po).max() <= 1e-12
            assert np.abs(fa - fd).max() <= 1e-12 * max(np.abs(fd).max(), 1.0), w
            assert np.abs(fa - fo).max() <= 1e-8 * max(np.abs(fo).max(), 1.0), w
        assert len(d.breaks()[0]) > 0  # the loading broke bonds on the way
    finally:
        sims["binding"].close()


def test_gravity_box_through_the_binding(makers):
    sims = {k: S.gravity_box(m, 6) for k, m in makers.items()}
    try:
        for s in sims.values():
            s.step(300)
        a, d, o = sims["binding"], sims["direct"], sims["oracle"]
        _compare(a, d, 1e-12, 1e-12, False)
        _compare(a, o, 1e-9, 1e-8, False)
        for w in ("zlo", "xlo"):
            fa, fo = a.wall(w)[1], o.wall(w)[1]
            assert np.abs(fa - fo).max() <= 1e-8 * max(np.abs(fo).max(), 1.0), w
        # unknown names: zero vectors and no effect, as the reference's workers answer
        p, f = a.wall("no_such_wall")
        assert not p.any() and not f.any()
    finally:
        sims["binding"].close()
