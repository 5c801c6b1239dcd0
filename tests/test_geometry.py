"""Set-up geometry (host only): the packers place non-overlapping spheres inside the box
with radii in range, the fitting packer is dense and connected, and the vectorised
distance connections equal a brute-force search."""
import numpy as np

from esys.lsm import geometry as G


def _overlaps(pos, rad):
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) - rad[:, None] - rad[None]
    np.fill_diagonal(d, np.inf)
    return d.min()


def test_fit_pack_is_dense_and_valid(dem_lib):
    pos, rad = G.fit_pack(3000, (0, 0, 0), (12, 12, 12), 0.3, 0.8, seed=3)
    assert len(rad) > 500
    assert _overlaps(pos, rad) >= -1e-8 * rad.max()
    assert (rad >= 0.3).all() and (rad <= 0.8).all()
    assert (pos - rad[:, None] >= -1e-9).all() and (pos + rad[:, None] <= 12 + 1e-9).all()
    frac = (4.0 / 3.0 * np.pi * rad ** 3).sum() / 12 ** 3
    pr, rr = G.rsi_pack(3000, (0, 0, 0), (12, 12, 12), uniform=(0.3, 0.8), rmin=0.3, rmax=0.8, seed=3,
                        max_attempts=200)
    assert frac > 0.45 and frac > (4.0 / 3.0 * np.pi * rr ** 3).sum() / 12 ** 3
    i, j = G.distance_connections(pos, rad, 1e-3)
    assert len(i) > 1.5 * len(rad)           # a load-bearing bonded solid


def test_distance_connections_equals_brute_force(dem_lib):
    pos, rad = G.rsi_pack(400, (0, 0, 0), (8, 8, 8), uniform=(0.3, 0.6), rmin=0.3, rmax=0.6, seed=1)
    i, j = G.distance_connections(pos, rad, 0.3)
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) - rad[:, None] - rad[None]
    bi, bj = np.nonzero(np.triu(d <= 0.3, 1))
    assert np.array_equal(i, bi) and np.array_equal(j, bj)


def test_reference_library_packer_equals_product_packer(dem_lib, oracle_libs):
    """The bench's reference arm builds its packing with the packer linked into the reference
    library; it must place exactly the product library's spheres."""
    import ctypes as C

    import pytest

    if not oracle_libs.available("ref"):
        pytest.skip("reference library not built")
    D = C.POINTER(C.c_double)
    f = dem_lib.lsm_pack_rsi
    f.argtypes = [C.c_ulonglong, C.c_int, D, D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_int, D, D]
    f.restype = C.c_int
    n = 3000
    pos, rad = np.zeros((n, 3)), np.zeros(n)
    lo, hi = np.zeros(3), np.array([30.0, 15.0, 30.0])
    k = f(7, n, lo.ctypes.data_as(D), hi.ctypes.data_as(D), 1, 1, 0.5, 0.25, 0.2, 1.0, 5000, pos.ctypes.data_as(D),
          rad.ctypes.data_as(D))
    pr, rr = oracle_libs.rsi_pack_ref(7, n, lo, hi, 1, 1, 0.5, 0.25, 0.2, 1.0, 5000)
    assert k == len(rr) > 2000
    assert np.array_equal(pos[:k], pr) and np.array_equal(rad[:k], rr)
