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
#include "dem_common.cuh"
#include "dem_laws.cuh"
#include "dem_tiled.cuh"

namespace dem {

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
      const double x0 = p.x;
      p.x -= g.Lx * floor((p.x - g.xmin) / g.Lx);
      if (p.x >= g.xmin + g.Lx) p.x -= g.Lx;  // rounding at the upper face
      P.buf[cur].pr[i] = p;
      P.cshift[i] += p.x - x0;  // CParticle::setCircular moves m_initpos with m_pos (Model/Particle.cpp:335-341)
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
  P.dbound[i] = 0.f;
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
template <class H>
__global__ void k_pairs_write(Grid g, Particles P, int cur, const int* cell_start, const int* cell_list, ExclDev ex,
                              const int* start, unsigned long long* keys, int kind, const unsigned long long* old_keys,
                              int old_n, const H* old_hist, H* hist) {
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
  // history: kind 0 none; 1 carried for persistent pairs (PIS_ED::update); 2 reset (a history-bearing
  // law in a PIS_NE storage, rebuilt from scratch at every rebuild)
  if (kind == 0) return;
  for (int k = s; k < s + n; ++k) {
    const int j = (int)(keys[k] & 0xffffffffu);
    H h{};
    if (kind == 1) {
      int p = lower_bound_key(old_keys, 0, old_n, keys[k]);
      if (p < old_n && old_keys[p] == keys[k]) {
        V x1 = xyz(pi), x2 = image_of(g, x1, xyz(P.buf[cur].pr[j]));
        if (friction_persistent(x1, pi.w, x2, P.buf[cur].pr[j].w)) h = old_hist[p];
      }
    }
    hist[k] = h;
  }
}

// Device bond hand-off: for every pair of a freshly built list, the bond that excludes it
// (an intact bond of an excluding group, TSubLattice::setExIG), (group << 28) | index, or -1.
__global__ void k_pairs_xbond(const unsigned long long* keys, int m, ExclDev ex, int* xbond) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const unsigned long long key = keys[k];
  int r = -1;
  for (int e = 0; e < ex.n && r < 0; ++e) {
    const int p = lower_bound_key(ex.keys[e], 0, ex.count[e], key);
    if (p < ex.count[e] && ex.keys[e][p] == key && ex.broken_step[e][p] == kBondAlive) r = (ex.group[e] << 28) | p;
  }
  xbond[k] = r;
}
void launch_pairs_xbond(const unsigned long long* keys, int m, const ExclDev& ex, int* xbond, cudaStream_t s) {
  if (m > 0) k_pairs_xbond<<<(m + 255) / 256, 256, 0, s>>>(keys, m, ex, xbond);
}

// Device bond hand-off: kAdjHeld on the adjacency entries of the pairs with an excluding bond,
// so the step tests a bit of the entry it already holds instead of loading xbond.
__global__ void k_adj_mark_held(int ne, const int* xbond, int2* adj) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int2 en = adj[e];
  en.y = (en.y & ~kAdjHeld) | (xbond[en.y & kAdjIndex] >= 0 ? kAdjHeld : 0);
  adj[e] = en;
}
void launch_adj_mark_held(int ne, const int* xbond, int2* adj, cudaStream_t s) {
  if (ne > 0) k_adj_mark_held<<<(ne + 255) / 256, 256, 0, s>>>(ne, xbond, adj);
}

// Wall candidates counted from the particles' flags; intact bonds counted from the break log.
__global__ void k_count_candidates(int n, const unsigned* pflags, int* ncand) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned pf = pflags[i];
  if (!(pf & PF_ALIVE)) return;
  const int c = __popc((pf >> PF_WALL_SHIFT) & 0xffu);
  if (c) atomicAdd(ncand, c);
}
void launch_count_candidates(int n, const unsigned* pflags, int* ncand, cudaStream_t s) {
  if (n > 0) k_count_candidates<<<(n + 255) / 256, 256, 0, s>>>(n, pflags, ncand);
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
template <class H>
__global__ void k_merge(const unsigned long long* A, const H* Ah, int m, const unsigned long long* B, int nb,
                        unsigned long long* out, H* outh, int kind) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) {
    // number of B elements strictly less than A[k]
    int lo = 0, hi = nb;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (B[mid] < A[k]) lo = mid + 1; else hi = mid; }
    out[k + lo] = A[k];
    if (kind != 0) outh[k + lo] = Ah[k];
  } else if (k < m + nb) {
    int b = k - m;
    // number of A elements <= B[b]
    int lo = 0, hi = m;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (A[mid] <= B[b]) lo = mid + 1; else hi = mid; }
    out[b + lo] = B[b];
    if (kind != 0) outh[b + lo] = H{};
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
  if (kind != 0) ohist[pos[k]] = hist[k];
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

// Mark slots alive again (dem_revive_particles); their cells, pairs and wall candidacy come
// from the neighbour search the host schedules next.
__global__ void k_set_alive(Particles P, int cnt, const int* slots) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < cnt) P.pflags[slots[r]] |= PF_ALIVE;
}

// Alive flag of every slot (the rows dem_get_particles returns).
__global__ void k_alive_flags(Particles P, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P.n) flags[i] = (P.pflags[i] & PF_ALIVE) ? 1 : 0;
}

// The alive particles' state as host rows (row = rank of the slot among alive slots, or the
// slot itself when rows is null): id, position, velocity, spin, quaternion, force and moment,
// each into its own array (null: not wanted).  A non-rotational particle reports zero spin
// and moment and the identity quaternion.
__global__ void k_pack_particles(Particles P, int cur, int rot, const int* rows, int* id, double* pos, double* vel,
                                 double* angvel, double* quat, double* force, double* moment) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n || !(P.pflags[i] & PF_ALIVE)) return;
  const int r = rows ? rows[i] : i;
  const ParticleBuf b = P.buf[cur];
  auto put3 = [&](double* dst, const double4& v, bool zero) {
    if (!dst) return;
    dst[3 * (size_t)r] = zero ? 0.0 : v.x;
    dst[3 * (size_t)r + 1] = zero ? 0.0 : v.y;
    dst[3 * (size_t)r + 2] = zero ? 0.0 : v.z;
  };
  if (id) id[r] = P.id[i];
  if (pos) put3(pos, b.pr[i], false);
  if (vel) put3(vel, b.vm[i], false);
  if (angvel) put3(angvel, b.wi[i], !rot);
  if (force) put3(force, P.force[i], false);
  if (moment) put3(moment, P.moment[i], !rot);
  if (quat) {
    const double4 q = rot ? b.qq[i] : make_double4(1.0, 0.0, 0.0, 0.0);
    quat[4 * (size_t)r] = q.x;
    quat[4 * (size_t)r + 1] = q.y;
    quat[4 * (size_t)r + 2] = q.z;
    quat[4 * (size_t)r + 3] = q.w;
  }
}

// Displacement check after a host-side move (TSubLattice::checkNeighbors).
__global__ void k_check_disp(Particles P, int cur, double half_alpha_sq, int* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  if (!(P.pflags[i] & PF_ALIVE)) return;
  double4 p = P.buf[cur].pr[i], o = P.oldpos[i];
  V d = mk(p.x - o.x, p.y - o.y, p.z - o.z);
  if (dot(d, d) > half_alpha_sq) atomicOr(ctrl, CTRL_REBUILD);
  // the bound the step kernels extend restarts from this distance (the subtraction's rounding
  // of positions up to ~1e3 is covered by the absolute margin)
  P.dbound[i] = __fadd_ru(__fmul_ru(__double2float_ru(sqrt(dot(d, d))), 1.0000005f), 1e-9f);
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
// CEWallInteractionGroup::applyForce (EWallInteractionGroup.hpp:93-164): servo
// iteration of one wall against its candidates' elastic contacts.  One block of
// kServoThreads.  Thread t owns the slots t, t + kServoThreads, ... (a fixed assignment,
// so the sums are reproducible): it first lists its candidates of wall w, in slot order,
// in its own segment of idx (offsets from a block scan of the counts), then every
// iteration visits only that segment instead of rescanning all slots.
// ---------------------------------------------------------------------------
constexpr int kServoThreads = 1024;

__global__ void __launch_bounds__(kServoThreads) k_wall_servo(Particles P, int cur, int w, WallDev* walls, double Fx,
                                                               double Fy, double Fz, int* idx) {
  __shared__ double red[32][4];
  __shared__ int s_wsum[32];
  __shared__ int s_done;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const unsigned cand = 1u << (PF_WALL_SHIFT + w), inner = 1u << (PF_INNER_SHIFT + w);
  // this thread's candidates: count, block exclusive scan, then list them
  int c = 0;
  for (int i = t; i < P.n; i += kServoThreads) {
    const unsigned pf = P.pflags[i];
    c += ((pf & PF_ALIVE) && (pf & cand)) ? 1 : 0;
  }
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_wsum[wid] = incl;
  if (t == 0) s_done = 0;
  __syncthreads();
  if (wid == 0) {
    int v = s_wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    s_wsum[lane] = v;  // inclusive over warps
  }
  __syncthreads();
  const int off = (wid ? s_wsum[wid - 1] : 0) + incl - c;
  int e = off;
  for (int i = t; i < P.n; i += kServoThreads) {
    const unsigned pf = P.pflags[i];
    if ((pf & PF_ALIVE) && (pf & cand)) idx[e++] = (pf & inner) ? (i | (int)0x80000000) : i;
  }
  // the fixed point (each thread reads back only what it wrote itself)
  const V Fv = mk(Fx, Fy, Fz);
  const double Fn = norm(Fv);
  const V O_f = Fv / Fn;
  WallDev* W = walls + w;
  const double4* pr = P.buf[cur].pr;
  int it = 0;
  while (!s_done) {
    const V o = mk(W->ox, W->oy, W->oz), n = mk(W->nx, W->ny, W->nz);
    const double kw = W->k;
    double kl = 0, fx = 0, fy = 0, fz = 0;
    for (int q = off; q < off + c; ++q) {
      const int code = idx[q];
      const double4 p = pr[code & 0x7fffffff];
      double f = 1.0;
      f *= 3.141592654 * p.w;
      const double mk_ = f * kw;
      double dist = dot(xyz(p) - o, n);
      if (dist < p.w) {
        kl += mk_;  // getStiffness
        if (code < 0) {
          V fi = -1.0 * (mk_ * (p.w - dist) * n);  // getForce
          V cc = dot(fi, O_f) * O_f;
          fx += cc.x; fy += cc.y; fz += cc.z;
        }
      }
    }
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
      kl += __shfl_down_sync(0xffffffffu, kl, o2);
      fx += __shfl_down_sync(0xffffffffu, fx, o2);
      fy += __shfl_down_sync(0xffffffffu, fy, o2);
      fz += __shfl_down_sync(0xffffffffu, fz, o2);
    }
    if (lane == 0) { red[wid][0] = kl; red[wid][1] = fx; red[wid][2] = fy; red[wid][3] = fz; }
    __syncthreads();
    if (t == 0) {
      double K = 0, gx = 0, gy = 0, gz = 0;
      for (int k = 0; k < kServoThreads / 32; ++k) { K += red[k][0]; gx += red[k][1]; gy += red[k][2]; gz += red[k][3]; }
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

// Block-local exclusive scan of one 8192-element chunk per block; the chunk total to bsum.
__global__ void k_scan_chunks(const int* in, int* out, int n, int* bsum) {
  __shared__ int warp_sums[32];
  const int T = blockDim.x;
  const int base = blockIdx.x * T * 8;
  int v[8];
  int local = 0;
  const int start = base + threadIdx.x * 8;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int idx = start + k;
    v[k] = idx < n ? in[idx] : 0;
    local += v[k];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = lane < (T >> 5) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_sums[lane] = t;
  }
  __syncthreads();
  int excl = (w > 0 ? warp_sums[w - 1] : 0) + x - local;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int idx = start + k;
    if (idx < n) out[idx] = excl;
    excl += v[k];
  }
  if (threadIdx.x == T - 1) bsum[blockIdx.x] = excl;
}

__global__ void k_scan_add(int* out, int n, const int* boff) {
  const int base = blockIdx.x * blockDim.x * 8;
  const int off = boff[blockIdx.x];
  for (int k = threadIdx.x; k < blockDim.x * 8; k += blockDim.x) {
    const int idx = base + k;
    if (idx < n) out[idx] += off;
  }
}

// Exclusive scan of n ints (in place allowed), total to *total.  Up to one
// 8192-element chunk: one block; beyond: chunk scans, a scan of the chunk totals
// (in tmp, >= chunks + 1 ints) and an offset pass.
void launch_scan(const int* in, int* out, int n, int* total, int* tmp, cudaStream_t s) {
  constexpr int kChunk = 1024 * 8;
  if (n <= kChunk || !tmp) {
    k_scan<<<1, 1024, 0, s>>>(in, out, n, total);
    return;
  }
  const int nb = (n + kChunk - 1) / kChunk;
  k_scan_chunks<<<nb, 1024, 0, s>>>(in, out, n, tmp);
  k_scan<<<1, 1024, 0, s>>>(tmp, tmp, nb, total);
  k_scan_add<<<nb, 1024, 0, s>>>(out, n, tmp);
}
int scan_tmp_ints(int n) { return (n + 8191) / 8192 + 1; }
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
template <class H>
void launch_pairs_write(const Grid& g, const Particles& P, int cur, const int* cs, const int* cl, const ExclDev& ex,
                        const int* start, unsigned long long* keys, int kind, const unsigned long long* old_keys,
                        int old_n, const H* old_hist, H* hist, cudaStream_t s) {
  if (P.n)
    k_pairs_write<H><<<nblk(P.n, 128), 128, 0, s>>>(g, P, cur, cs, cl, ex, start, keys, kind, old_keys, old_n,
                                                     old_hist, hist);
}
template void launch_pairs_write<double4>(const Grid&, const Particles&, int, const int*, const int*, const ExclDev&,
                                          const int*, unsigned long long*, int, const unsigned long long*, int,
                                          const double4*, double4*, cudaStream_t);
template void launch_pairs_write<float4>(const Grid&, const Particles&, int, const int*, const int*, const ExclDev&,
                                         const int*, unsigned long long*, int, const unsigned long long*, int,
                                         const float4*, float4*, cudaStream_t);
void launch_adj(const unsigned long long* keys, int m, int n, int* adj_count, int* p1_start, int* adj_start,
                int* adj_cursor, int2* adj, int* total, int* tmp, cudaStream_t s) {
  cudaMemsetAsync(adj_count, 0, sizeof(int) * (n + 1), s);
  cudaMemsetAsync(adj_cursor, 0, sizeof(int) * (n + 1), s);
  int t = (m > n + 1 ? m : n + 1);
  k_adj_count<<<nblk(t, 256), 256, 0, s>>>(keys, m, n, adj_count, p1_start);
  if (n) k_adj_add_p1<<<nblk(n, 256), 256, 0, s>>>(n, p1_start, adj_count);
  launch_scan(adj_count, adj_start, n + 1, total, tmp, s);
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
template <class H>
void launch_merge(const unsigned long long* A, const H* Ah, int m, const unsigned long long* B, int nb,
                  unsigned long long* out, H* outh, int kind, cudaStream_t s) {
  if (m + nb) k_merge<H><<<nblk(m + nb, 256), 256, 0, s>>>(A, Ah, m, B, nb, out, outh, kind);
}
template void launch_merge<double4>(const unsigned long long*, const double4*, int, const unsigned long long*, int,
                                    unsigned long long*, double4*, int, cudaStream_t);
template void launch_merge<float4>(const unsigned long long*, const float4*, int, const unsigned long long*, int,
                                   unsigned long long*, float4*, int, cudaStream_t);

// FP32 copies of velocity and spin for the FP32-force form (one 32-byte record per particle).
__global__ void k_sync_vw(Particles P, int cur) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const double4 v = P.buf[cur].vm[i], w = P.buf[cur].wi[i];
  P.buf[cur].vw[2 * i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)w.x);
  P.buf[cur].vw[2 * i + 1] = make_float4((float)w.y, (float)w.z, 0.f, 0.f);
}
void launch_sync_vw(const Particles& P, int cur, cudaStream_t s) {
  if (P.n) k_sync_vw<<<nblk(P.n, 256), 256, 0, s>>>(P, cur);
}

// History conversion when the precision form changes (FP64 <-> FP32 records).
__global__ void k_hist_to_f32(int m, const double4* in, float4* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) { double4 h = in[k]; out[k] = make_float4((float)h.x, (float)h.y, (float)h.z, (float)h.w); }
}
__global__ void k_hist_to_f64(int m, const float4* in, double4* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) { float4 h = in[k]; out[k] = make_double4(h.x, h.y, h.z, h.w); }
}
void launch_hist_convert(int m, const double4* d, float4* f, bool to_f32, cudaStream_t s) {
  if (!m) return;
  if (to_f32) k_hist_to_f32<<<nblk(m, 256), 256, 0, s>>>(m, d, f);
  else k_hist_to_f64<<<nblk(m, 256), 256, 0, s>>>(m, f, const_cast<double4*>(d));
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
void launch_set_alive(const Particles& P, int cnt, const int* slots, cudaStream_t s) {
  if (cnt) k_set_alive<<<nblk(cnt, 256), 256, 0, s>>>(P, cnt, slots);
}
void launch_alive_flags(const Particles& P, int* flags, cudaStream_t s) {
  if (P.n) k_alive_flags<<<nblk(P.n, 256), 256, 0, s>>>(P, flags);
}
void launch_pack_particles(const Particles& P, int cur, int rot, const int* rows, int* id, double* pos, double* vel,
                           double* angvel, double* quat, double* force, double* moment, cudaStream_t s) {
  if (P.n)
    k_pack_particles<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, rot, rows, id, pos, vel, angvel, quat, force, moment);
}
void launch_check_disp(const Particles& P, int cur, double half_alpha_sq, int* ctrl, cudaStream_t s) {
  if (P.n) k_check_disp<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, half_alpha_sq, ctrl);
}
void launch_move_tagged(const Particles& P, int cur, int tag, const double* d, cudaStream_t s) {
  if (P.n) k_move_tagged<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, tag, d[0], d[1], d[2]);
}
void launch_wall_servo(const Particles& P, int cur, int w, WallDev* walls, const double* F, int* idx, cudaStream_t s) {
  k_wall_servo<<<1, kServoThreads, 0, s>>>(P, cur, w, walls, F[0], F[1], F[2], idx);
}

int step_grid(int n, int tpp) { return step_blocks(n, tpp); }

// FP64 instances (this translation unit is built with --fmad=false).
// The bond pass of both precision forms, built here without FMA contraction: the RotBond law's
// acos of a cosine near 1 turns a last-bit difference into ~1e-8 rad, so a contracted build
// would not reproduce the FP64 form's bond forces.
void launch_bond_pass_f64(const StepArgs& a, bool eval, cudaStream_t s) {
  if (eval) launch_bond_pass<true, false>(a, s);
  else launch_bond_pass<false, false>(a, s);
}

// PIS_EB::update of BrittleBeamSC groups at the head of a step (BrittleBeamSCInteraction::broken,
// Model/BrittleBeamSC.cpp:96-150): the positions the step starts from and the stress sums of the step
// before.  A failure removes the bond before this step's forces and stops the chunk, so that the host's
// update builds the new pairs first (as updateInteractions does after a bond update); the relaunched
// step finds the bond gone.  Bonds of group d only; the event's step is the step that opens with it.
__global__ void k_sc_check(const StepArgs a, int d, int nb) {
  if (*a.stop) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const BondDev& B = a.bond[d];
  const long long step = *a.step_counter + 1;
  if (B.broken_step[k] <= step) return;
  const ParticleBuf in = a.P.buf[a.cur];
  const int2 e = B.ends[k];
  const double4 pa = in.pr[e.x], pb = in.pr[e.y];
  const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
  if (!sc_broken(x1, pa.w, a.sig + 9 * (size_t)e.x, x2, pb.w, a.sig + 9 * (size_t)e.y, B.cohesion, B.tan_angle,
                 B.t_cutoff))
    return;
  B.broken_step[k] = (int)step;
  a.P.flagged[e.x] = 1;
  a.P.flagged[e.y] = 1;
  if (!a.replay) {
    const int slot = atomicAdd(B.nevents, 1);
    if (slot < B.cap_events) {
      B.events[3 * slot] = a.P.id[e.x];
      B.events[3 * slot + 1] = a.P.id[e.y];
      B.events[3 * slot + 2] = (int)step;
    } else {
      atomicOr(a.ctrl, CTRL_OVERFLOW);
    }
    atomicOr(a.ctrl, CTRL_BROKE);
  }
  if (a.handoff) a.brk_step[(step - 1) & 1] = (int)(step - 1);
  else *a.stop = 1;
}

void launch_step(const StepArgs& a, bool rot, int tpp, bool split, cudaStream_t s) {
  bool el = false, fr = false, widened = false;
  for (int d = 0; d < a.ndyn; ++d) {
    if (a.dyn[d].kind >= 2) widened = true;  // NRotFriction, HertzMindlin
    (a.dyn[d].kind == 0 ? el : fr) = true;
  }
  for (int d = 0; d < a.nbond; ++d) widened = widened || a.bond[d].kind == 1 || a.bond[d].kind == 3;
  const bool bd = a.nbond > 0;
  const bool gather = bd && a.bond[0].bf;  // bonds evaluated once by the bond pass
  if (a.sig)
    for (int d = 0; d < a.nbond; ++d)
      if (a.bond[d].kind == 3 && a.bond[d].nb_launch > 0)
        k_sc_check<<<(a.bond[d].nb_launch + kBondPassThreads - 1) / kBondPassThreads, kBondPassThreads, 0, s>>>(
            a, d, a.bond[d].nb_launch);
  if (gather) launch_bond_pass<false, false>(a, s);
  if (widened && a.sig && rot)  // BrittleBeamSC: the general instance with the stress sums
    return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_NFRIC | F_BGATHER | F_STRESS, false, false>(a, tpp, s);
  if (widened) {  // NRotFriction / HertzMindlin / NRotBond groups: one general instance per particle type
    if (!rot) return launch_step_tpp<false, F_ELASTIC | F_NFRIC | F_BGATHER, false, false>(a, tpp, s);
    return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_NFRIC | F_BGATHER, false, false>(a, tpp, s);
  }
  if (split) {
    if (!rot) return launch_split_tpp<false, F_ELASTIC, false>(a, tpp, s);
    if (!bd && fr && !el) return launch_split_tpp<true, F_FRIC, false>(a, tpp, s);
    if (!bd && !fr) return launch_split_tpp<true, F_ELASTIC, false>(a, tpp, s);
    if (gather) return launch_split_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, false>(a, tpp, s);
    if (bd && !el) return launch_split_tpp<true, F_FRIC | F_BOND, false>(a, tpp, s);
    return launch_split_tpp<true, F_ELASTIC | F_FRIC | F_BOND, false>(a, tpp, s);
  }
  if (!rot) return launch_step_tpp<false, F_ELASTIC, false, false>(a, tpp, s);
  if (!bd && fr && !el) return launch_step_tpp<true, F_FRIC, false, false>(a, tpp, s);
  if (!bd && !fr) return launch_step_tpp<true, F_ELASTIC, false, false>(a, tpp, s);
  if (gather && !el) return launch_step_tpp<true, F_FRIC | F_BGATHER, false, false>(a, tpp, s);
  if (gather) return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, false, false>(a, tpp, s);
  if (bd && !el) return launch_step_tpp<true, F_FRIC | F_BOND, false, false>(a, tpp, s);
  return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BOND, false, false>(a, tpp, s);
}

}  // namespace dem

namespace dem {

// ---------------------------------------------------------------------------
// Field savers: per-particle and per-interaction scalar fields, computed on the
// device (operation order of the reference's accessors, this unit being built
// without FMA contraction).  Dead slots get NaN and are skipped by the host.
// ---------------------------------------------------------------------------
// CParticle::getKineticEnergy etc. (Model/Particle.h:116,134; Model/RotParticle.h:198-200)
__global__ void k_particle_field(Particles P, int cur, int rot, int field, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  if (!(P.pflags[i] & PF_ALIVE)) { out[i] = __longlong_as_double(0x7ff8000000000000LL); return; }
  const double4 p = P.buf[cur].pr[i], vm = P.buf[cur].vm[i];
  const V v = xyz(vm);
  double r = 0.0;
  switch (field) {
    case 0: {  // e_kin
      if (rot) {
        const double4 wi = P.buf[cur].wi[i];
        const V w = xyz(wi);
        r = (0.5 * vm.w) * dot(v, v) + dot((0.5 * wi.w) * w, w);
      } else {
        r = dot((0.5 * vm.w) * v, v);
      }
      break;
    }
    case 1: r = rot ? (0.5 * vm.w) * dot(v, v) : dot((0.5 * vm.w) * v, v); break;  // e_kin_linear
    case 2: { const double4 wi = P.buf[cur].wi[i]; const V w = xyz(wi); r = rot ? dot((0.5 * wi.w) * w, w) : 0.0; break; }
    case 3: r = norm(v); break;                                                     // v_abs
    case 4: r = p.w; break;                                                         // radius
    case 5: r = (double)P.id[i]; break;                                             // id
    case 6: r = (double)P.tag[i]; break;                                            // tag
    default: r = vm.w; break;                                                       // mass
  }
  out[i] = r;
}
void launch_particle_field(const Particles& P, int cur, int rot, int field, double* out, cudaStream_t s) {
  if (P.n) k_particle_field<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, rot, field, out);
}

// Per-particle vector fields (CParticle::getVectorFieldFunction, Model/Particle.cpp:166-184;
// CRotParticle's, Model/RotParticle.cpp:459-480): 0 position, 1 velocity, 2 force, 3 ang_velocity
// (getAngVelNR), 4 displacement (getTotalDisplacement = m_pos - m_initpos, m_initpos carried
// along by the circular shifts).  initpos: 3 doubles per slot, the position at creation.
__global__ void k_particle_vector_field(Particles P, int cur, int field, const double* initpos, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  V r = mk(0.0, 0.0, 0.0);
  switch (field) {
    case 0: r = xyz(P.buf[cur].pr[i]); break;
    case 1: r = xyz(P.buf[cur].vm[i]); break;
    case 2: r = xyz(P.force[i]); break;
    case 3: r = xyz(P.buf[cur].wi[i]); break;
    default: {
      const V x = xyz(P.buf[cur].pr[i]);
      const V x0 = mk(initpos[3 * i] + P.cshift[i], initpos[3 * i + 1], initpos[3 * i + 2]);
      r = x - x0;
    }
  }
  out[3 * i] = r.x;
  out[3 * i + 1] = r.y;
  out[3 * i + 2] = r.z;
}
void launch_particle_vector_field(const Particles& P, int cur, int field, const double* initpos, double* out,
                                  cudaStream_t s) {
  if (P.n) k_particle_vector_field<<<nblk(P.n, 256), 256, 0, s>>>(P, cur, field, initpos, out);
}

// Pair fields of a dynamic group from the state its last force evaluation read (buffer `prev`)
// and the history it wrote: field 0 count, 1 potential_energy, 2 slipping, 3 sticking
// (CElasticInteraction, Model/ElasticInteraction.cpp:76-96; CRotFrictionInteraction,
// Model/RotFricInteraction.cpp:384-452).
template <class H>
__global__ void k_pair_field(Grid g, Particles P, int prev, const unsigned long long* keys, int m, int kind,
                             double k, double ks, int scaling, int meanR, const H* hist, int field, double* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const int s1 = (int)(keys[q] >> 32), s2 = (int)(keys[q] & 0xffffffffu);
  const double4 pa = P.buf[prev].pr[s1], pb = P.buf[prev].pr[s2];
  const V x1 = xyz(pa), x2 = image_of(g, x1, xyz(pb));
  const V D = x1 - x2;
  const double d2 = dot(D, D), eq = pa.w + pb.w;
  double r = 0.0;
  if (kind == 0) {
    const bool touching = d2 < eq * eq;
    if (field == 0) r = touching ? 1.0 : 0.0;
    else if (field == 1 && touching) {
      const double ke = elastic_k(k, scaling, pa.w, pb.w);
      const double dist = sqrt(d2);
      const V F = D * (ke * (dist - eq) / dist);
      r = dot(0.5 * F, F) / ke;
    }
  } else {
    const H h = hist[q];
    const int fl = (int)h.w;
    const bool touching = (fl & 2) != 0, slipping = (fl & 1) != 0;
    if (field == 0) r = touching ? 1.0 : 0.0;
    else if (field == 2) r = slipping ? 1.0 : 0.0;
    else if (field == 3) r = (touching && !slipping) ? 1.0 : 0.0;
    else if (field == 1 && touching && (kind == 3 || kind == 4)) {
      // CHertzMindlinInteraction::getPotentialEnergy (HertzMindlinInteraction.cpp:371-375) and
      // CHertzMindlinViscoInteraction::getPotentialEnergy (HertzMindlinViscoInteraction.cpp:415-419):
      // the elastic Hertz normal force, the damping left out
      const double R_ij = 1.0 / (1.0 / pa.w + 1.0 / pb.w);
      const double dist = sqrt(d2);
      const double dn = eq - dist;
      const V fn = (D / norm(D)) * (4.0 / 3.0 * k * sqrt(R_ij) * pow(dn, 1.5));
      r = dot(0.5 * fn, fn) / k;  // k holds E
    } else if (field == 1 && touching) {
      // CRotFrictionInteraction / CFrictionInteraction::getPotentialEnergy (FrictionInteraction.cpp:336-342)
      double ke, kse;
      if (kind == 2) nfriction_k(k, ks, scaling, pa.w, pb.w, ke, kse);
      else friction_k(k, ks, scaling, meanR, pa.w, pb.w, ke, kse);
      const double dist = sqrt(d2);
      const V Fn = D * (ke * (dist - eq) / dist);
      const V Ff = mk((double)h.x, (double)h.y, (double)h.z);
      r = dot(0.5 * Fn, Fn) / ke + dot(0.5 * Ff, Ff) / kse;
    }
  }
  out[q] = r;
}
void launch_pair_field(const Grid& g, const Particles& P, int prev, const unsigned long long* keys, int m, int kind,
                       double k, double ks, int scaling, int meanR, const double4* hist, const float4* hist32,
                       int field, double* out, cudaStream_t s) {
  if (m <= 0) return;
  if (hist32) k_pair_field<float4><<<nblk(m, 256), 256, 0, s>>>(g, P, prev, keys, m, kind, k, ks, scaling, meanR, hist32, field, out);
  else k_pair_field<double4><<<nblk(m, 256), 256, 0, s>>>(g, P, prev, keys, m, kind, k, ks, scaling, meanR, hist, field, out);
}

// Bond fields from the state the last force evaluation read: 0 count, 1 potential_energy,
// 2 e_pot_normal, 3 e_pot_shear, 4 e_pot_twist, 5 e_pot_bend, 6 breaking_criterion
// (ARotBondedInteraction.cpp:456-485, CRotBondedInteraction::getCriterion :221-227).  NaN for
// bonds removed before that evaluation.
__global__ void k_bond_field(Grid g, Particles P, int prev, long long t, BondDev B, int nb, int field, double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  if (B.broken_step[k] <= t) { out[k] = __longlong_as_double(0x7ff8000000000000LL); return; }
  if (field == 0) { out[k] = 1.0; return; }
  const int2 e = B.ends[k];
  const double4 pa = P.buf[prev].pr[e.x], pb = P.buf[prev].pr[e.y], qa = P.buf[prev].qq[e.x], qb = P.buf[prev].qq[e.y];
  const V x1 = xyz(pa), x2 = image_of(g, x1, xyz(pb));
  const V mD = xyz(B.D0[k]);
  const double dist0 = sqrt(dot(mD, mD));
  const BondK K = bond_k(B.kr, B.ks, B.kt, B.kb, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, pa.w, pb.w);
  BondOut o;
  law_bond(K, mD, x1, pa.w, Qd{qa.x, mk(qa.y, qa.z, qa.w)}, x2, pb.w, Qd{qb.x, mk(qb.y, qb.z, qb.w)}, o);
  const double pr = (K.kr != 0.0) ? 0.5 * (o.nF * o.nF) / K.kr : 0.0;
  const double ps = (K.ks != 0.0) ? 0.5 * (o.shF * o.shF) / K.ks : 0.0;
  const double pt = (K.kt != 0.0) ? 0.5 * (o.tM * o.tM) / K.kt : 0.0;
  const double pb_ = (K.kb != 0.0) ? 0.5 * (o.bM * o.bM) / K.kb : 0.0;
  double r;
  switch (field) {
    case 1: r = pr + ps + pt + pb_; break;
    case 2: r = pr; break;
    case 3: r = ps; break;
    case 4: r = pt; break;
    case 5: r = pb_; break;
    default: r = o.nF / K.max_n + o.shF / K.max_s + o.tM / K.max_t + o.bM / K.max_b; break;
  }
  out[k] = r;
}
void launch_bond_field(const Grid& g, const Particles& P, int prev, long long t, const BondDev& B, int nb, int field,
                       double* out, cudaStream_t s) {
  if (nb > 0) k_bond_field<<<nblk(nb, 256), 256, 0, s>>>(g, P, prev, t, B, nb, field, out);
}

}  // namespace dem
