// Device helpers shared by the DEM kernels: the reference's cell indexing,
// periodic images, the neighbour-list predicate, key search and read-only loads.
#pragma once
#include "dem_device.cuh"
#include "dem_laws.cuh"

namespace dem {

__device__ __forceinline__ int cell_coord(double x, double p0, double dim, int g) {
  return int(floor((x - p0) / dim)) - g;  // NeighborTable::index (ntable.hpp:128-140)
}

// Cell of a position, -1 when outside the local table.  Periodic x wraps.
__device__ __forceinline__ int cell_of(const Grid& g, double x, double y, double z) {
  if (!(isfinite(x) && isfinite(y) && isfinite(z))) return -1;
  int ix = cell_coord(x, g.p0x, g.dim, g.gx);
  int iy = cell_coord(y, g.p0y, g.dim, g.gy);
  int iz = cell_coord(z, g.p0z, g.dim, g.gz);
  if (g.circx) ix = ((ix % g.nx) + g.nx) % g.nx;
  if (ix >= 0 && ix < g.nx && iy >= 0 && iy < g.ny && iz >= 0 && iz < g.nz) return (ix * g.ny + iy) * g.nz + iz;
  return -1;
}

// NeighborTable::isInInner (ntable.hpp:212-233).
__device__ __forceinline__ bool inner_of(const Grid& g, double x, double y, double z) {
  int ix = cell_coord(x, g.p0x, g.dim, g.gx);
  int iy = cell_coord(y, g.p0y, g.dim, g.gy);
  int iz = cell_coord(z, g.p0z, g.dim, g.gz);
  bool inx = g.circx ? true : (ix > 0 && ix < g.nx - 1);
  if (g.nz < 3) return inx && iy > 0 && iy < g.ny - 1;
  return inx && iy > 0 && iy < g.ny - 1 && iz > 0 && iz < g.nz - 1;
}

// Position of p2 as seen from p1: its periodic image nearest p1.
__device__ __forceinline__ V image_of(const Grid& g, const V& x1, V x2) {
  if (g.circx) {
    double dx = x1.x - x2.x;
    if (dx > 0.5 * g.Lx) x2.x += g.Lx;
    else if (dx < -0.5 * g.Lx) x2.x -= g.Lx;
  }
  return x2;
}

// Neighbour-list predicate of NeighborTable::addPairsToList (ntable.hpp:471-489),
// evaluated in canonical orientation (lo = lower id).
__device__ __forceinline__ bool near_pair(const Grid& g, const double4& plo, const double4& phi) {
  V xl = xyz(plo), xh = image_of(g, xl, xyz(phi));
  double dist2 = norm2(xl - xh);
  double dmax = plo.w + phi.w + g.alpha;
  return dist2 <= (dmax * dmax);
}

// Visit the particles of the 27 cells around cell c (wrapping x when periodic).
template <class F>
__device__ __forceinline__ void for_neighbour_cells(const Grid& g, int c, const int* cell_start, const int* cell_list,
                                                    F&& f) {
  const int iz = c % g.nz, iy = (c / g.nz) % g.ny, ix = c / (g.nz * g.ny);
  for (int dx = -1; dx <= 1; ++dx) {
    int jx = ix + dx;
    if (g.circx) jx = (jx + g.nx) % g.nx;
    else if (jx < 0 || jx >= g.nx) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      int jy = iy + dy;
      if (jy < 0 || jy >= g.ny) continue;
      for (int dz = -1; dz <= 1; ++dz) {
        int jz = iz + dz;
        if (jz < 0 || jz >= g.nz) continue;
        int cc = (jx * g.ny + jy) * g.nz + jz;
        for (int k = cell_start[cc]; k < cell_start[cc + 1]; ++k) f(cell_list[k]);
      }
    }
  }
}

// 32-byte read-only gather through the non-coherent (texture) path.  Only for
// arrays the running kernel does not write (the step's input buffer).
__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Bring a line into L1 without holding registers (records a kernel reads later).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
// Programmatic dependent launch (sm_90+): wait for the prerequisite grid's completion and memory
// (returns at once for a grid launched without a programmatic dependency), and allow the
// dependent grid to launch.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ unsigned long long pair_key(int a, int b) {
  return ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
}

// Lower bound of key in sorted keys[lo, hi).
__device__ __forceinline__ int lower_bound_key(const unsigned long long* keys, int lo, int hi, unsigned long long key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool has_key(const unsigned long long* keys, int n, unsigned long long key) {
  int p = lower_bound_key(keys, 0, n, key);
  return p < n && keys[p] == key;
}

// An intact bond of an excluding group with this (p1 slot, p2 slot) key?
__device__ __forceinline__ bool excluded(const ExclDev& ex, unsigned long long key) {
  for (int e = 0; e < ex.n; ++e) {
    int p = lower_bound_key(ex.keys[e], 0, ex.count[e], key);
    if (p < ex.count[e] && ex.keys[e][p] == key && ex.broken_step[e][p] == kBondAlive) return true;
  }
  return false;
}

}  // namespace dem
