// CUDA kernels of the DEM step for sm_100a (FP64 path; built with --fmad=false
// so every + - * / sqrt rounds like the reference's x86-64 double arithmetic).
//
//  k_step<ROT,TPP>     one timestep for all particles: walls, gravity, pair
//                      groups, bonds, damping, integration, displacement check.
//                      TPP lanes per particle stride over the particle's
//                      adjacency and combine with a fixed-order butterfly, so
//                      results are run-to-run bit-reproducible; no atomics on
//                      forces.  Replaces TSubLattice::oneStep + checkNeighbors
//                      (Parallel/SubLattice.hpp:2066-2236, 2473-2519).
//  k_bin ... k_adj_*   the neighbour search / interaction update
//                      (ntable/src/ntable.hpp:262-664, pis/pi_storage_ne.hpp:49-102,
//                      pis/pi_storage_ed.hpp:84-161).
#include <climits>
#include <cstdio>

#include "dem_device.cuh"
#include "dem_kernels.h"
#include "dem_laws.cuh"

namespace dem {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
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

// Single-block exclusive scan of n ints (in place allowed); total written to *total.
__global__ void k_scan(const int* in, int* out, int n, int* total) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int T = blockDim.x;
  for (int base = 0; base < n; base += T * 8) {
    int v[8];
    int local = 0;
    const int start = base + threadIdx.x * 8;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      int idx = start + k;
      v[k] = idx < n ? in[idx] : 0;
      local += v[k];
    }
    // inclusive scan of `local` across the block
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
      int s = lane < (T >> 5) ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    int excl = carry + (w > 0 ? warp_sums[w - 1] : 0) + x - local;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      int idx = start + k;
      if (idx < n) out[idx] = excl;
      excl += v[k];
    }
    __syncthreads();
    if (threadIdx.x == T - 1) carry = excl;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// ---------------------------------------------------------------------------
// neighbour search: NeighborTable::build (ntable.hpp:262-288) + resetDisplacements
// ---------------------------------------------------------------------------
__global__ void k_bin(Grid g, Particles P, int cur, int* cell_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  unsigned pf = P.pflags[i];
  if (!(pf & PF_ALIVE)) { P.cell[i] = -1; return; }
  double4 p = P.buf[cur].pr[i];
  if (g.circx && isfinite(p.x)) {  // circular shift of particles that left through an x face (pp_array.hpp:465-503)
    if (p.x >= g.xmin + g.Lx || p.x < g.xmin) {
      p.x -= g.Lx * floor((p.x - g.xmin) / g.Lx);
      if (p.x >= g.xmin + g.Lx) p.x -= g.Lx;  // rounding at the upper face
      P.buf[cur].pr[i] = p;
    }
  }
  int c = cell_of(g, p.x, p.y, p.z);
  if (c < 0) {  // outside the table: the particle is deleted (ntable.hpp:281-286)
    P.pflags[i] = pf & ~PF_ALIVE;
    P.cell[i] = -1;
    return;
  }
  P.cell[i] = c;
  P.oldpos[i] = make_double4(p.x, p.y, p.z, 0.0);
  atomicAdd(&cell_count[c], 1);
}

__global__ void k_scatter_cells(Particles P, const int* cell_start, int* cell_cursor, int* cell_list) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int c = P.cell[i];
  if (c < 0) return;
  int k = atomicAdd(&cell_cursor[c], 1);
  cell_list[cell_start[c] + k] = i;
}

// Order each cell's particles by slot (the reference's list order).
__global__ void k_sort_cells(int ncell, const int* cell_start, int* cell_list) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int s = cell_start[c], e = cell_start[c + 1];
  for (int a = s + 1; a < e; ++a) {
    int v = cell_list[a];
    int b = a - 1;
    while (b >= s && cell_list[b] > v) { cell_list[b + 1] = cell_list[b]; --b; }
    cell_list[b + 1] = v;
  }
}

// ---------------------------------------------------------------------------
// full pair list of a dynamic group (getFullList + PIS_NE/PIS_ED::update)
// ---------------------------------------------------------------------------
// Count, per particle i, the neighbours j with id[j] > id[i] within the cutoff
// that are not excluded.
__global__ void k_pairs_count(Grid g, Particles P, int cur, const int* cell_start, const int* cell_list, ExclDev ex,
                              int* count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int c = P.cell[i];
  if (c < 0) { count[i] = 0; return; }
  const double4 pi = P.buf[cur].pr[i];
  const int idi = P.id[i];
  int n = 0;
  for_neighbour_cells(g, c, cell_start, cell_list, [&](int j) {
    if (P.id[j] <= idi) return;
    if (!near_pair(g, pi, P.buf[cur].pr[j])) return;
    if (ex.n && excluded(ex, pair_key(i, j))) return;
    ++n;
  });
  count[i] = n;
}

// Write the pairs (p1 = i) into [start[i], start[i]+count[i]) sorted by p2 slot
// and carry RotFriction history from the previous list when the old
// interaction is persistent (PIS_ED::update, pi_storage_ed.hpp:93-128).
__global__ void k_pairs_write(Grid g, Particles P, int cur, const int* cell_start, const int* cell_list, ExclDev ex,
                              const int* start, unsigned long long* keys, int kind, const unsigned long long* old_keys,
                              int old_n, const double4* old_hist, double4* hist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int c = P.cell[i];
  if (c < 0) return;
  const double4 pi = P.buf[cur].pr[i];
  const int idi = P.id[i];
  const int s = start[i];
  int n = 0;
  for_neighbour_cells(g, c, cell_start, cell_list, [&](int j) {
    if (P.id[j] <= idi) return;
    if (!near_pair(g, pi, P.buf[cur].pr[j])) return;
    unsigned long long key = pair_key(i, j);
    if (ex.n && excluded(ex, key)) return;
    // insertion into the sorted segment
    int b = s + n - 1;
    while (b >= s && keys[b] > key) { keys[b + 1] = keys[b]; --b; }
    keys[b + 1] = key;
    ++n;
  });
  if (kind != 1) return;
  for (int k = s; k < s + n; ++k) {
    const int j = (int)(keys[k] & 0xffffffffu);
    double4 h = make_double4(0.0, 0.0, 0.0, 0.0);
    int p = lower_bound_key(old_keys, 0, old_n, keys[k]);
    if (p < old_n && old_keys[p] == keys[k]) {
      V x1 = xyz(pi), x2 = image_of(g, x1, xyz(P.buf[cur].pr[j]));
      if (friction_persistent(x1, pi.w, x2, P.buf[cur].pr[j].w)) h = old_hist[p];
    }
    hist[k] = h;
  }
}

// ---------------------------------------------------------------------------
// adjacency (both directions) from a key-sorted pair list
// ---------------------------------------------------------------------------
__global__ void k_adj_count(const unsigned long long* keys, int m, int n, int* adj_count, int* p1_start) {
  // p1_start[i] = first pair with p1 == i (keys are sorted by p1 slot)
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p1_start[i] = lower_bound_key(keys, 0, m, (unsigned long long)(unsigned)i << 32);
  if (i == n) p1_start[n] = m;
  int k = i;
  if (k < m) atomicAdd(&adj_count[(int)(keys[k] & 0xffffffffu)], 1);
}

__global__ void k_adj_add_p1(int n, const int* p1_start, int* adj_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) adj_count[i] += p1_start[i + 1] - p1_start[i];
}

__global__ void k_adj_fill(const unsigned long long* keys, int m, const int* p1_start, const int* adj_start,
                           int* adj_cursor, int2* adj) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  int a = (int)(keys[k] >> 32), b = (int)(keys[k] & 0xffffffffu);
  // p1 role: entries first, in key order
  adj[adj_start[a] + (k - p1_start[a])] = make_int2(b, k | (int)0x80000000);
  // p2 role: after b's p1 entries, order fixed by a sort below
  int off = (p1_start[b + 1] - p1_start[b]) + atomicAdd(&adj_cursor[b], 1);
  adj[adj_start[b] + off] = make_int2(a, k);
}

__global__ void k_adj_sort(int n, const int* p1_start, const int* adj_start, int2* adj) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = adj_start[i] + (p1_start[i + 1] - p1_start[i]), e = adj_start[i + 1];
  for (int a = s + 1; a < e; ++a) {
    int2 v = adj[a];
    int b = a - 1;
    while (b >= s && adj[b].y > v.y) { adj[b + 1] = adj[b]; --b; }
    adj[b + 1] = v;
  }
}

// ---------------------------------------------------------------------------
// "new list" after bond breaks (NeighborTable::getNewList, ntable.hpp:532-583,
// 628-664): pairs of two flagged particles in the same or adjacent cells of the
// last build, no distance test.
// ---------------------------------------------------------------------------
__global__ void k_newlist_count(Grid g, Particles P, const int* cell_start, const int* cell_list, ExclDev ex,
                                const unsigned long long* keys, int m, int check_in, int* count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int c = P.cell[i];
  if (c < 0 || !P.flagged[i]) { count[i] = 0; return; }
  const int idi = P.id[i];
  int n = 0;
  for_neighbour_cells(g, c, cell_start, cell_list, [&](int j) {
    if (P.id[j] <= idi || !P.flagged[j]) return;
    unsigned long long key = pair_key(i, j);
    if (ex.n && excluded(ex, key)) return;
    if (check_in && has_key(keys, m, key)) return;
    ++n;
  });
  count[i] = n;
}

__global__ void k_newlist_write(Grid g, Particles P, const int* cell_start, const int* cell_list, ExclDev ex,
                                const unsigned long long* keys, int m, int check_in, const int* start,
                                unsigned long long* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int c = P.cell[i];
  if (c < 0 || !P.flagged[i]) return;
  const int idi = P.id[i];
  const int s = start[i];
  int n = 0;
  for_neighbour_cells(g, c, cell_start, cell_list, [&](int j) {
    if (P.id[j] <= idi || !P.flagged[j]) return;
    unsigned long long key = pair_key(i, j);
    if (ex.n && excluded(ex, key)) return;
    if (check_in && has_key(keys, m, key)) return;
    int b = s + n - 1;
    while (b >= s && out[b] > key) { out[b + 1] = out[b]; --b; }
    out[b + 1] = key;
    ++n;
  });
}

// Merge sorted lists A (m, with history) and B (nb new pairs, fresh history);
// equal keys keep A first (stable), as the reference appends new interactions.
__global__ void k_merge(const unsigned long long* A, const double4* Ah, int m, const unsigned long long* B, int nb,
                        unsigned long long* out, double4* outh, int kind) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) {
    // number of B elements strictly less than A[k]
    int lo = 0, hi = nb;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (B[mid] < A[k]) lo = mid + 1; else hi = mid; }
    out[k + lo] = A[k];
    if (kind == 1) outh[k + lo] = Ah[k];
  } else if (k < m + nb) {
    int b = k - m;
    // number of A elements <= B[b]
    int lo = 0, hi = m;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (A[mid] <= B[b]) lo = mid + 1; else hi = mid; }
    out[b + lo] = B[b];
    if (kind == 1) outh[b + lo] = make_double4(0.0, 0.0, 0.0, 0.0);
  }
}

__global__ void k_clear_flags(int n, unsigned char* flagged) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flagged[i] = 0;
}

// Erase pairs whose particles vanished (PIS_E::rebuild, pi_storage_e.hpp:111-155):
// mark them, then compact with a scan.
__global__ void k_pairs_alive(const unsigned long long* keys, int m, const unsigned* pflags, int* keep) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  int a = (int)(keys[k] >> 32), b = (int)(keys[k] & 0xffffffffu);
  keep[k] = ((pflags[a] & PF_ALIVE) && (pflags[b] & PF_ALIVE)) ? 1 : 0;
}

__global__ void k_compact(const unsigned long long* keys, const double4* hist, int m, const int* keep, const int* pos,
                          unsigned long long* okeys, double4* ohist, int kind) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m || !keep[k]) return;
  okeys[pos[k]] = keys[k];
  if (kind == 1) ohist[pos[k]] = hist[k];
}

// Bonds whose particle vanished are erased (PIS_E::rebuild); no break event.
__global__ void k_bonds_rebuild(int nb, const int2* ends, const unsigned* pflags, int* broken_step) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int2 e = ends[b];
  if (!((pflags[e.x] & PF_ALIVE) && (pflags[e.y] & PF_ALIVE))) broken_step[b] = 0;
}

// m_D = pos(p2) - pos(p1) at bond creation (ARotBondedInteraction ctor, ARotBondedInteraction.cpp:149).
__global__ void k_bonds_init(int nb, const int2* ends, const double4* pr, double4* D0) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int2 e = ends[b];
  double4 a = pr[e.x], c = pr[e.y];
  D0[b] = make_double4(c.x - a.x, c.y - a.y, c.z - a.z, 0.0);
}

// Wall candidates (CEWallInteractionGroup::Update, EWallInteractionGroup.hpp:57-82;
// getParticlesAtPlane, ntable.hpp:674-690).
__global__ void k_wall_update(Grid g, Particles P, int cur, int nwall, const WallDev* walls, int* ncand) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  unsigned pf = P.pflags[i] & ~(0xffffu << PF_WALL_SHIFT);
  if (pf & PF_ALIVE) {
    double4 p = P.buf[cur].pr[i];
    bool inner = inner_of(g, p.x, p.y, p.z);
    for (int w = 0; w < nwall; ++w) {
      const WallDev& W = walls[w];
      V x = mk(p.x, p.y, p.z), o = mk(W.ox, W.oy, W.oz), n = mk(W.nx, W.ny, W.nz);
      double dist = dot(x - o, n);
      if (fabs(dist) < g.dim) {
        pf |= 1u << (PF_WALL_SHIFT + w);
        if (inner) pf |= 1u << (PF_INNER_SHIFT + w);
      }
    }
    const int c = __popc((pf >> PF_WALL_SHIFT) & 0xffu);
    if (c) atomicAdd(ncand, c);
  }
  P.pflags[i] = pf;
}

// Bulk state upload (dem_set_particles): rows -> slots, radius / mass / inertia kept.
__global__ void k_set_state(Particles P, int cur, int cnt, const int* slots, const double* pos, const double* vel,
                            const double* angvel, const double* quat) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= cnt) return;
  int i = slots ? slots[r] : r;
  ParticleBuf b = P.buf[cur];
  if (pos) { double4 p = b.pr[i]; p.x = pos[3 * r]; p.y = pos[3 * r + 1]; p.z = pos[3 * r + 2]; b.pr[i] = p; }
  if (vel) { double4 v = b.vm[i]; v.x = vel[3 * r]; v.y = vel[3 * r + 1]; v.z = vel[3 * r + 2]; b.vm[i] = v; }
  if (angvel) { double4 w = b.wi[i]; w.x = angvel[3 * r]; w.y = angvel[3 * r + 1]; w.z = angvel[3 * r + 2]; b.wi[i] = w; }
  if (quat) b.qq[i] = make_double4(quat[4 * r], quat[4 * r + 1], quat[4 * r + 2], quat[4 * r + 3]);
}

// Displacement check after a host-side move (TSubLattice::checkNeighbors).
__global__ void k_check_disp(Particles P, int cur, double half_alpha_sq, int* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  if (!(P.pflags[i] & PF_ALIVE)) return;
  double4 p = P.buf[cur].pr[i], o = P.oldpos[i];
  V d = mk(p.x - o.x, p.y - o.y, p.z - o.z);
  if (dot(d, d) > half_alpha_sq) atomicOr(ctrl, CTRL_REBUILD);
}

// moveTaggedParticlesBy (SubLattice.hpp:2577-2587): exact tag match.
__global__ void k_move_tagged(Particles P, int cur, int tag, double dx, double dy, double dz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  if (!(P.pflags[i] & PF_ALIVE) || P.tag[i] != tag) return;
  double4 p = P.buf[cur].pr[i];
  p.x += dx; p.y += dy; p.z += dz;
  P.buf[cur].pr[i] = p;
}

// ---------------------------------------------------------------------------
// the timestep
// ---------------------------------------------------------------------------
template <int TPP>
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
  for (int o = 1; o < TPP; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int TPP>
__device__ __forceinline__ V lane_sum(V v) {
  return mk(lane_sum<TPP>(v.x), lane_sum<TPP>(v.y), lane_sum<TPP>(v.z));
}

constexpr int kStepThreads = 256;
constexpr int kStepWarps = kStepThreads / 32;

// Interaction families compiled into a k_step instance (the host picks the
// smallest instance that covers the groups present, so a friction-only run
// does not carry the registers of the bond law).
enum : int { F_ELASTIC = 1, F_FRIC = 2, F_BOND = 4 };

template <bool ROT, int TPP, int FEAT>
__global__ void __launch_bounds__(kStepThreads, (FEAT & F_BOND) ? 1 : 2) k_step(const StepArgs a) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  if (*a.stop) return;  // an earlier step of this chunk asked the host to intervene
  const long long step = *a.step_counter + 1;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / TPP;
  const int lane = threadIdx.x % TPP;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool valid = i < a.P.n;
  const unsigned pf = valid ? a.P.pflags[i] : 0u;
  const bool alive = valid && (pf & PF_ALIVE);
  const ParticleBuf in = a.P.buf[a.cur];
  const ParticleBuf out = a.P.buf[a.cur ^ 1];

  double4 p4 = make_double4(0, 0, 0, 0), v4 = p4, w4 = p4, q4 = make_double4(1, 0, 0, 0);
  if (alive) {
    p4 = in.pr[i];
    v4 = in.vm[i];
    if (ROT) {
      w4 = in.wi[i];
      if (FEAT & F_BOND) q4 = in.qq[i];
    }
  }
  const V xi = xyz(p4);
  V F = mk(0.0, 0.0, 0.0), M = mk(0.0, 0.0, 0.0);

  // 1. elastic walls, in group-name order (TSubLattice::calcForces, SubLattice.hpp:2116-2120).
  //    The walls' reactions are reduced in a fixed order: warp shuffle, then warps, then blocks.
  for (int w = 0; w < a.nwall; ++w) {
    V c = mk(0.0, 0.0, 0.0);
    if (alive && lane == 0 && (pf & (1u << (PF_WALL_SHIFT + w)))) {
      const WallDev W = a.walls[w];
      V f;
      if (law_wall(W.k, mk(W.ox, W.oy, W.oz), mk(W.nx, W.ny, W.nz), xi, p4.w, f)) {
        F += f;
        if (pf & (1u << (PF_INNER_SHIFT + w))) c = f;  // CWall::addForce(-F): m_force -= -F
      }
    }
    double cx = c.x, cy = c.y, cz = c.z;
    if (__any_sync(0xffffffffu, cx != 0.0 || cy != 0.0 || cz != 0.0)) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        cx += __shfl_down_sync(0xffffffffu, cx, o);
        cy += __shfl_down_sync(0xffffffffu, cy, o);
        cz += __shfl_down_sync(0xffffffffu, cz, o);
      }
    }
    if (wlane == 0) { s_red[warp][w][0] = cx; s_red[warp][w][1] = cy; s_red[warp][w][2] = cz; }
  }

  // 2. body forces (BodyForceGroup::calcForces, BodyForceGroup.hpp:54-65): F += g * m
  if (alive && lane == 0)
    for (int k = 0; k < a.ngrav; ++k) F += mk(a.grav[k][0], a.grav[k][1], a.grav[k][2]) * v4.w;

  // 3. dynamic pair groups (PIS_NE / PIS_ED::calcForces)
  V Fp = mk(0.0, 0.0, 0.0), Mp = mk(0.0, 0.0, 0.0);
  if ((FEAT & (F_ELASTIC | F_FRIC)) && alive) {
    for (int d = 0; d < a.ndyn; ++d) {
      const DynDev& G = a.dyn[d];
      const int e0 = G.adj_start[i], e1 = G.adj_start[i + 1];
      for (int e = e0 + lane; e < e1; e += TPP) {
        const int2 en = G.adj[e];
        const int j = en.x;
        const bool isp1 = en.y < 0;
        const int k = en.y & 0x7fffffff;
        const double4 pj = in.pr[j];
        // canonical orientation: p1 = lower id
        const double4 pa = isp1 ? p4 : pj, pb = isp1 ? pj : p4;
        const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
        if (G.kind == 0) {
          if constexpr ((FEAT & F_ELASTIC) != 0) {
            V f;
            if (law_elastic(elastic_k(G.k, G.scaling, pa.w, pb.w), x1, pa.w, x2, pb.w, f)) {
              if (isp1) Fp += -1.0 * f; else Fp += f;
            }
          }
        } else {
          if constexpr (ROT && (FEAT & F_FRIC) != 0) {
            const double4 vj = in.vm[j], wj = in.wi[j];
            const double4 va = isp1 ? v4 : vj, vb = isp1 ? vj : v4;
            const double4 wa = isp1 ? w4 : wj, wb = isp1 ? wj : w4;
            const double4 h = G.hist_in[k];
            double keff, kseff;
            friction_k(G.k, G.ks, G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
            FricOut o;
            law_friction(keff, kseff, G.mu_s, G.mu_d, G.dt, x1, pa.w, xyz(va), xyz(wa), x2, pb.w, xyz(vb), xyz(wb),
                         mk(h.x, h.y, h.z), (((int)h.w) & 1) != 0, o);
            if (isp1) {
              Fp += -1.0 * o.fn;
              Mp += o.M1;
              Fp += o.Ffric;
              G.hist_out[k] = make_double4(o.Ffric.x, o.Ffric.y, o.Ffric.z,
                                           (o.slipping ? 1.0 : 0.0) + (o.touching ? 2.0 : 0.0));
            } else {
              Fp += o.fn;
              Mp += o.M2;
              Fp += -1.0 * o.Ffric;
            }
          }
        }
      }
    }
  }

  // 4. bonded groups (PIS_EB::calcForces) + failure test (PIS_EB::update at the next step)
  V Fb = mk(0.0, 0.0, 0.0), Mb = mk(0.0, 0.0, 0.0);
  if constexpr (ROT && (FEAT & F_BOND) != 0) {
    if (alive) {
      for (int d = 0; d < a.nbond; ++d) {
        const BondDev& B = a.bond[d];
        const int e0 = B.adj_start[i], e1 = B.adj_start[i + 1];
        for (int e = e0 + lane; e < e1; e += TPP) {
          const int2 en = B.adj[e];
          const int k = en.y & 0x7fffffff;
          if (B.broken_step[k] <= step) continue;  // removed by an earlier update
          const int j = en.x;
          const bool isp1 = en.y < 0;
          const double4 pj = in.pr[j], qj = in.qq[j];
          const double4 pa = isp1 ? p4 : pj, pb = isp1 ? pj : p4;
          const double4 qa = isp1 ? q4 : qj, qb = isp1 ? qj : q4;
          const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
          const double4 D0 = B.D0[k];
          const V mD = xyz(D0);
          const double dist0 = sqrt(dot(mD, mD));
          const BondK K = bond_k(B.kr, B.ks, B.kt, B.kb, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, pa.w, pb.w);
          BondOut o;
          law_bond(K, mD, x1, pa.w, Qd{qa.x, mk(qa.y, qa.z, qa.w)}, x2, pb.w, Qd{qb.x, mk(qb.y, qb.z, qb.w)}, o);
          if (isp1) {
            Fb += o.force;
            Mb += o.moment1;
            if (bond_broken(K, o, B.truncated)) {
              B.broken_step[k] = (int)(step + 1);
              a.P.flagged[i] = 1;
              a.P.flagged[j] = 1;
              int slot = atomicAdd(B.nevents, 1);
              if (slot < B.cap_events) {
                B.events[3 * slot] = a.P.id[i];
                B.events[3 * slot + 1] = a.P.id[j];
                B.events[3 * slot + 2] = (int)(step + 1);
              } else {
                atomicOr(a.ctrl, CTRL_OVERFLOW);
              }
              atomicOr(a.ctrl, CTRL_BROKE);
            }
          } else {
            Fb += -1.0 * o.force;
            Mb += o.moment2;
          }
        }
      }
    }
  }

  // fixed-order combination of the lanes' partial sums
  if (TPP > 1) {
    Fp = lane_sum<TPP>(Fp);
    Mp = lane_sum<TPP>(Mp);
    if (FEAT & F_BOND) {
      Fb = lane_sum<TPP>(Fb);
      Mb = lane_sum<TPP>(Mb);
    }
  }

  if (alive && lane == 0) {
    F += Fp;
    M += Mp;
    F += Fb;
    M += Mb;
    const double2 iv = a.P.inv[i];
    // 5. damping, last (SubLattice.hpp:2140-2145): "Damping" then "RotDamping"
    if (a.damp_lin) F += damping_force(xyz(v4), F, iv.x, v4.w, a.visc_lin, a.dt_lin, a.iter_lin);
    if (ROT && a.damp_rot) M += damping_force(xyz(w4), M, iv.y, w4.w, a.visc_rot, a.dt_rot, a.iter_rot);
    // 6. integration (CRotParticle::integrate + rescale, RotParticle.cpp:277-321; Particle.cpp:257-274)
    const double dt = a.dt;
    V v = xyz(v4), x = xi;
    if (ROT) {
      if (!(FEAT & F_BOND)) q4 = in.qq[i];
      V w = xyz(w4);
      Qd q{q4.x, mk(q4.y, q4.z, q4.w)};
      if (pf & PF_ROT) {
        w += (dt * iv.y) * M;
        const Qd dq = qmul(Qd{0.0, w}, q);
        const double c = dt / 2.0;
        q.s += c * dq.s;
        q.v += c * dq.v;
      } else {
        w = mk(0.0, 0.0, 0.0);
      }
      const double module = sqrt(q.s * q.s + q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z);
      if (module != 0.0) {
        const double inverse = 1.0 / module;
        q.s = inverse * q.s;
        q.v = inverse * q.v;
      }
      out.wi[i] = d4(w, w4.w);
      out.qq[i] = make_double4(q.s, q.v.x, q.v.y, q.v.z);
    }
    if (pf & PF_DYN) {
      v += F * iv.x * dt;
      x += v * dt;
    }
    out.pr[i] = d4(x, p4.w);
    out.vm[i] = d4(v, v4.w);
    if (a.store_forces) {
      a.P.force[i] = d4(F, 0.0);
      if (ROT) a.P.moment[i] = d4(M, 0.0);
    }
    // 7. displacement check for the next step (TSubLattice::checkNeighbors)
    const double4 op = a.P.oldpos[i];
    const V dd = mk(x.x - op.x, x.y - op.y, x.z - op.z);
    if (dot(dd, dd) > a.half_alpha_sq) atomicOr(a.ctrl, CTRL_REBUILD);
  }

  // per-block wall reactions (fixed order over warps), then the last block finishes the step
  const int nw3 = a.nwall * 3;
  __syncthreads();
  if (threadIdx.x < nw3) {
    const int w = threadIdx.x / 3, c = threadIdx.x % 3;
    double acc = 0.0;
    for (int k = 0; k < kStepWarps; ++k) acc += s_red[k][w][c];
    a.wall_partial[((size_t)blockIdx.x * kMaxWalls + w) * 3 + c] = acc;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicInc(a.block_counter, gridDim.x - 1);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // wall reactions: thread t sums blocks t, t+256, ... (fixed assignment), then a fixed tree
  for (int wc = 0; wc < nw3; ++wc) {
    const int w = wc / 3, c = wc % 3;
    double acc = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      acc += __ldcg(a.wall_partial + ((size_t)b * kMaxWalls + w) * 3 + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (wlane == 0) s_red[warp][0][0] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < kStepWarps; ++k) t += s_red[k][0][0];
      a.wall_force[3 * w + c] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int w = 0; w < a.nwall; ++w) {  // native wall loader: origin += v*dt per step (WallLoaderRunnable)
      WallDev* W = a.walls + w;
      if (a.wall_vel[3 * w] != 0.0 || a.wall_vel[3 * w + 1] != 0.0 || a.wall_vel[3 * w + 2] != 0.0) {
        W->ox += a.wall_vel[3 * w] * a.dt;
        W->oy += a.wall_vel[3 * w + 1] * a.dt;
        W->oz += a.wall_vel[3 * w + 2] * a.dt;
      }
    }
    *a.step_counter = step;
    volatile int* ctrl = a.ctrl;
    if (*ctrl) *a.stop = 1;
  }
}

// ---------------------------------------------------------------------------
// CEWallInteractionGroup::applyForce (EWallInteractionGroup.hpp:93-164): servo
// iteration of one wall against its candidates' elastic contacts.  One block.
// ---------------------------------------------------------------------------
__global__ void k_wall_servo(Particles P, int cur, int w, WallDev* walls, double Fx, double Fy, double Fz) {
  __shared__ double red[32][4];
  __shared__ double s_move[3];
  __shared__ int s_done;
  const V Fv = mk(Fx, Fy, Fz);
  const double Fn = norm(Fv);
  const V O_f = Fv / Fn;
  WallDev* W = walls + w;
  int it = 0;
  if (threadIdx.x == 0) s_done = 0;
  __syncthreads();
  while (!s_done) {
    const V o = mk(W->ox, W->oy, W->oz), n = mk(W->nx, W->ny, W->nz);
    double kl = 0, fx = 0, fy = 0, fz = 0;
    for (int i = threadIdx.x; i < P.n; i += blockDim.x) {
      unsigned pf = P.pflags[i];
      if (!(pf & PF_ALIVE) || !(pf & (1u << (PF_WALL_SHIFT + w)))) continue;
      const double4 p = P.buf[cur].pr[i];
      double f = 1.0;
      f *= 3.141592654 * p.w;
      const double mk_ = f * W->k;
      double dist = dot(xyz(p) - o, n);
      if (dist < p.w) {
        kl += mk_;  // getStiffness
        if (pf & (1u << (PF_INNER_SHIFT + w))) {
          V fi = -1.0 * (mk_ * (p.w - dist) * n);  // getForce
          V c = dot(fi, O_f) * O_f;
          fx += c.x; fy += c.y; fz += c.z;
        }
      }
    }
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
      kl += __shfl_down_sync(0xffffffffu, kl, o2);
      fx += __shfl_down_sync(0xffffffffu, fx, o2);
      fy += __shfl_down_sync(0xffffffffu, fy, o2);
      fz += __shfl_down_sync(0xffffffffu, fz, o2);
    }
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5][0] = kl; red[threadIdx.x >> 5][1] = fx; red[threadIdx.x >> 5][2] = fy; red[threadIdx.x >> 5][3] = fz; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double K = 0, gx = 0, gy = 0, gz = 0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { K += red[k][0]; gx += red[k][1]; gy += red[k][2]; gz += red[k][3]; }
      double d, ef;
      if (K > 0) {
        const V Fg = mk(gx, gy, gz);
        const double df = dot(Fv + Fg, O_f);
        d = df / K;
        ef = df / Fn;
      } else {
        d = 1e-5;
        ef = 1;
      }
      const V mv = d * O_f;
      W->ox += mv.x; W->oy += mv.y; W->oz += mv.z;
      ++it;
      s_done = !((it < 50) && (ef > 1e-3));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
static inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

void launch_scan(const int* in, int* out, int n, int* total, cudaStream_t s) {
  k_scan<<<1, 1024, 0, s>>>(in, out, n, total);
}
void launch_bin(const Grid& g, const Particles& P, int cur, int* cell_count, cudaStream_t s) {
  if (P.n) k_bin<<<nblk(P.n, 256), 256, 0, s>>>(g, P, cur, cell_count);
}
void launch_scatter_cells(const Particles& P, const int* cell_start, int* cursor, int* cell_list, cudaStream_t s) {
  if (P.n) k_scatter_cells<<<nblk(P.n, 256), 256, 0, s>>>(P, cell_start, cursor, cell_list);
}
void launch_sort_cells(int ncell, const int* cell_start, int* cell_list, cudaStream_t s) {
  k_sort_cells<<<nblk(ncell, 256), 256, 0, s>>>(ncell, cell_start, cell_list);
}
void launch_pairs_count(const Grid& g, const Particles& P, int cur, const int* cs, const int* cl, const ExclDev& ex,
                        int* count, cudaStream_t s) {
  if (P.n) k_pairs_count<<<nblk(P.n, 128), 128, 0, s>>>(g, P, cur, cs, cl, ex, count);
}
void launch_pairs_write(const Grid& g, const Particles& P, int cur, const int* cs, const int* cl, const ExclDev& ex,
                        const int* start, unsigned long long* keys, int kind, const unsigned long long* old_keys,
                        int old_n, const double4* old_hist, double4* hist, cudaStream_t s) {
  if (P.n)
    k_pairs_write<<<nblk(P.n, 128), 128, 0, s>>>(g, P, cur, cs, cl, ex, start, keys, kind, old_keys, old_n, old_hist,
                                                  hist);
}
void launch_adj(const unsigned long long* keys, int m, int n, int* adj_count, int* p1_start, int* adj_start,
                int* adj_cursor, int2* adj, int* total, cudaStream_t s) {
  cudaMemsetAsync(adj_count, 0, sizeof(int) * (n + 1), s);
  cudaMemsetAsync(adj_cursor, 0, sizeof(int) * (n + 1), s);
  int t = (m > n + 1 ? m : n + 1);
  k_adj_count<<<nblk(t, 256), 256, 0, s>>>(keys, m, n, adj_count, p1_start);
  if (n) k_adj_add_p1<<<nblk(n, 256), 256, 0, s>>>(n, p1_start, adj_count);
  k_scan<<<1, 1024, 0, s>>>(adj_count, adj_start, n + 1, total);
  if (m) k_adj_fill<<<nblk(m, 256), 256, 0, s>>>(keys, m, p1_start, adj_start, adj_cursor, adj);
  if (n) k_adj_sort<<<nblk(n, 256), 256, 0, s>>>(n, p1_start, adj_start, adj);
}
void launch_newlist_count(const Grid& g, const Particles& P, const int* cs, const int* cl, const ExclDev& ex,
                          const unsigned long long* keys, int m, int check_in, int* count, cudaStream_t s) {
  if (P.n) k_newlist_count<<<nblk(P.n, 128), 128, 0, s>>>(g, P, cs, cl, ex, keys, m, check_in, count);
}
void launch_newlist_write(const Grid& g, const Particles& P, const int* cs, const int* cl, const ExclDev& ex,
                          const unsigned long long* keys, int m, int check_in, const int* start,
                          unsigned long long* out, cudaStream_t s) {
  if (P.n) k_newlist_write<<<nblk(P.n, 128), 128, 0, s>>>(g, P, cs, cl, ex, keys, m, check_in, start, out);
}
void launch_merge(const unsigned long long* A, const double4* Ah, int m, const unsigned long long* B, int nb,
                  unsigned long long* out, double4* outh, int kind, cudaStream_t s) {
  if (m + nb) k_merge<<<nblk(m + nb, 256), 256, 0, s>>>(A, Ah, m, B, nb, out, outh, kind);
}
void launch_clear_flags(int n, unsigned char* flagged, cudaStream_t s) {
  if (n) k_clear_flags<<<nblk(n, 256), 256, 0, s>>>(n, flagged);
}
void launch_pairs_alive(const unsigned long long* keys, int m, const unsigned* pflags, int* keep, cudaStream_t s) {
  if (m) k_pairs_alive<<<nblk(m, 256), 256, 0, s>>>(keys, m, pflags, keep);
}
void launch_compact(const unsigned long long* keys, const double4* hist, int m, const int* keep, const int* pos,
                    unsigned long long* okeys, double4* ohist, int kind, cudaStream_t s) {
  if (m) k_compact<<<nblk(m, 256), 256, 0, s>>>(keys, hist, m, keep, pos, okeys, ohist, kind);
}
void launch_bonds_rebuild(int nb, const int2* ends, const unsigned* pflags, int* broken_step, cudaStream_t s) {
  if (nb) k_bonds_rebuild<<<nblk(nb, 256), 256, 0, s>>>(nb, ends, pflags, broken_step);
}
void launch_bonds_init(int nb, const int2* ends, const double4* pr, double4* D0, cudaStream_t s) {
  if (nb) k_bonds_init<<<nblk(nb, 256), 256, 0, s>>>(nb, ends, pr, D0);
}
void launch_wall_update(const Grid& g, const Particles& P, int cur, int nwall, const WallDev* walls, int* ncand,
                        cudaStream_t s) {
  if (P.n) k_wall_update<<<nblk(P.n, 256), 256, 0, s>>>(g, P, cur, nwall, walls, ncand);
}
void launch_set_state(const Particles& P, int cur, int cnt, const int* slots, const double* pos, const double* vel,
                      const double* angvel, const double* quat, cudaStream_t s) {
  if (cnt) k_set_state<<<nblk(cnt, 256), 256, 0, s>>>(P, cur, cnt, slots, pos, vel, angvel, quat);
}
void launch_check_disp(const Particles& P, int cur, double half_alpha_sq, int* ctrl, cudaStream_t s) {
  if (P.n) k_check_disp<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, half_alpha_sq, ctrl);
}
void launch_move_tagged(const Particles& P, int cur, int tag, const double* d, cudaStream_t s) {
  if (P.n) k_move_tagged<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, tag, d[0], d[1], d[2]);
}
void launch_wall_servo(const Particles& P, int cur, int w, WallDev* walls, const double* F, cudaStream_t s) {
  k_wall_servo<<<1, 1024, 0, s>>>(P, cur, w, walls, F[0], F[1], F[2]);
}

int step_grid(int n, int tpp) { return nblk((long long)(n > 0 ? n : 1) * tpp, kStepThreads); }

template <bool R, int FEAT>
static void launch_step_tpp(const StepArgs& a, int tpp, int grid, cudaStream_t s) {
  switch (tpp) {
    case 1: k_step<R, 1, FEAT><<<grid, kStepThreads, 0, s>>>(a); break;
    case 2: k_step<R, 2, FEAT><<<grid, kStepThreads, 0, s>>>(a); break;
    case 4: k_step<R, 4, FEAT><<<grid, kStepThreads, 0, s>>>(a); break;
    default: k_step<R, 8, FEAT><<<grid, kStepThreads, 0, s>>>(a); break;
  }
}

void launch_step(const StepArgs& a, bool rot, int tpp, cudaStream_t s) {
  const int grid = step_grid(a.P.n, tpp);
  bool el = false, fr = false;
  for (int d = 0; d < a.ndyn; ++d) (a.dyn[d].kind == 0 ? el : fr) = true;
  const bool bd = a.nbond > 0;
  if (!rot) return launch_step_tpp<false, F_ELASTIC>(a, tpp, grid, s);
  if (!bd && fr && !el) return launch_step_tpp<true, F_FRIC>(a, tpp, grid, s);
  if (!bd && !fr) return launch_step_tpp<true, F_ELASTIC>(a, tpp, grid, s);
  if (bd && !el) return launch_step_tpp<true, F_FRIC | F_BOND>(a, tpp, grid, s);
  return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BOND>(a, tpp, grid, s);
}

}  // namespace dem
