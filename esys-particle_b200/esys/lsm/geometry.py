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
        lib.lsm_dist_connections.argtypes = [C.c_int, _D, _D, C.c_double, C.c_longlong, C.POINTER(C.c_int),
                                             C.POINTER(C.c_int)]
        lib.lsm_dist_connections.restype = C.c_longlong
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
    (Geometry/DistConnections.hpp), sorted by (i, j); the library's cell-grid search."""
    pos = np.ascontiguousarray(pos, np.float64)
    rad = np.ascontiguousarray(rad, np.float64)
    n = len(rad)
    lib = _lib()
    I = C.POINTER(C.c_int)
    cap = 8 * n
    while True:
        a, b = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        m = lib.lsm_dist_connections(n, pos.ctypes.data_as(_D), rad.ctypes.data_as(_D), float(max_gap), cap,
                                     a.ctypes.data_as(I), b.ctypes.data_as(I))
        if m < 0:
            raise ValueError("bad connection arguments")
        if m <= cap:
            return a[:m].astype(np.int64), b[:m].astype(np.int64)
        cap = int(m)
