"""Seeded synthetic packings and bond connectivity for set-up scripts and benchmarks.

Stand-ins for the reference's set-up geometry (Geometry/RandomBoxPacker.hpp,
Geometry/DistConnections.hpp, the Python ``RandomBoxPacker`` and
``ConnectionFinder``): host code only, not part of the per-step path.  The
packers are the library's (include/esys_geometry.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi

_D = C.POINTER(C.c_double)

__all__ = ["rsi_pack", "fit_pack", "distance_connections"]


def _lib():
    lib = _capi.load_library()
    if not getattr(lib, "_geometry_bound", False):
        lib.lsm_pack_rsi.argtypes = [C.c_ulonglong, C.c_int, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_int, _D, _D]
        lib.lsm_pack_rsi.restype = C.c_int
        lib.lsm_pack_fit.argtypes = [C.c_ulonglong, C.c_int, _D, _D, C.c_double, C.c_double, C.c_int, _D, _D]
        lib.lsm_pack_fit.restype = C.c_int
        lib._geometry_bound = True
    return lib


def rsi_pack(n, bmin, bmax, seed=0, periodic_x=False, lognormal=None, uniform=None, rmin=0.2, rmax=1.0,
             max_attempts=5000):
    """Random sequential insertion of up to n spheres; radii lognormal (median, sigma) or
    uniform (lo, hi), clipped to [rmin, rmax].  Returns (pos [m, 3], rad [m])."""
    dist, (p0, p1) = (1, lognormal) if lognormal is not None else (0, uniform or (rmin, rmax))
    pos, rad = np.zeros((n, 3)), np.zeros(n)
    lo, hi = np.asarray(bmin, np.float64), np.asarray(bmax, np.float64)
    m = _lib().lsm_pack_rsi(seed, n, lo.ctypes.data_as(_D), hi.ctypes.data_as(_D), int(periodic_x), dist,
                            float(p0), float(p1), float(rmin), float(rmax), int(max_attempts),
                            pos.ctypes.data_as(_D), rad.ctypes.data_as(_D))
    if m < 0:
        raise ValueError("bad packing arguments")
    return pos[:m].copy(), rad[:m].copy()


def fit_pack(n, bmin, bmax, rmin=0.2, rmax=1.0, seed=0, max_failures=2000):
    """Dense packing by gap filling (spheres fitted to their nearest neighbours and the box
    faces), up to n spheres with radii in [rmin, rmax].  Returns (pos [m, 3], rad [m])."""
    pos, rad = np.zeros((n, 3)), np.zeros(n)
    lo, hi = np.asarray(bmin, np.float64), np.asarray(bmax, np.float64)
    m = _lib().lsm_pack_fit(seed, n, lo.ctypes.data_as(_D), hi.ctypes.data_as(_D), float(rmin), float(rmax),
                            int(max_failures), pos.ctypes.data_as(_D), rad.ctypes.data_as(_D))
    if m < 0:
        raise ValueError("bad packing arguments")
    return pos[:m].copy(), rad[:m].copy()


def distance_connections(pos, rad, max_gap):
    """Pairs (i, j), i < j, whose gap |x_i - x_j| - r_i - r_j is at most max_gap
    (Geometry/DistConnections.hpp), vectorised over a cell sort."""
    pos = np.asarray(pos, np.float64)
    rad = np.asarray(rad, np.float64)
    n = len(rad)
    if n < 2:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    cell = 2.0 * rad.max() + max_gap
    key3 = np.floor((pos - pos.min(0)) / cell).astype(np.int64)
    dims = key3.max(0) + 3
    lin = lambda k: (k[:, 0] * dims[1] + k[:, 1]) * dims[2] + k[:, 2]
    key3 = key3 + 1
    keys = lin(key3)
    order = np.argsort(keys, kind="stable")
    sk = keys[order]
    out_i, out_j = [], []
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                nk = lin(key3 + np.array([dx, dy, dz]))
                lo = np.searchsorted(sk, nk, "left")
                hi = np.searchsorted(sk, nk, "right")
                cnt = hi - lo
                if cnt.sum() == 0:
                    continue
                src = np.repeat(np.arange(n), cnt)
                off = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
                dst = order[np.repeat(lo, cnt) + off]
                keep = src < dst
                src, dst = src[keep], dst[keep]
                gap = np.linalg.norm(pos[src] - pos[dst], axis=1) - rad[src] - rad[dst]
                ok = gap <= max_gap
                out_i.append(src[ok])
                out_j.append(dst[ok])
    i = np.concatenate(out_i)
    j = np.concatenate(out_j)
    o = np.lexsort((j, i))
    return i[o], j[o]
