// Tiled step kernels: the block-cooperative form of k_step and k_step_batch.
//
// A block takes a tile of kTileThreads consecutive particle slots, one thread per
// particle for the particle's own work.  The tile's entries of a group's
// per-particle adjacency form one contiguous range of that CSR, so the block
// reads the range coalesced and spreads its entries evenly over its threads:
// every thread then has several independent partner gathers in flight, instead
// of one lane walking one particle's entries through a chain of dependent loads
// (adjacency start -> entry -> partner record).  Each entry's contribution (the
// force and moment on the entry's own particle) goes to shared memory; the
// particle's own thread then adds its entries in adjacency order, which is the
// order of a one-lane k_step, so the sums are fixed-order and bit-reproducible
// with no atomics.  Walls, body forces, damping, integration and the epilogue are
// k_step's own (finish_particle, step_epilogue / batch_tile_epilogue).
//
// The pair laws, their orientation (p1 = lower id, evaluated from both sides at
// one call site) and the history writes (p1 side only) are those of pair_sums in
// dem_step.cuh (TSubLattice::calcForces over PIS_NE / PIS_ED groups,
// Parallel/SubLattice.hpp:2109-2154; CElasticInteraction::calcForces,
// Model/ElasticInteraction.cpp:54-71; CRotFrictionInteraction::calcSimpleForces,
// Model/RotFricInteraction.cpp:171-231).  Instances with the widened laws, in-line
// bonds or stress sums keep the lane-parallel kernels.
#pragma once
#include <type_traits>

#include "dem_step.cuh"

namespace dem {

template <int FEAT>
struct TiledSupported {
  static constexpr bool value = (FEAT & (F_NFRIC | F_BOND | F_STRESS)) == 0;
};

// Launch shape of the tiled kernels (compile-time; the defaults are the measured best on
// B200): resident blocks per SM targeted by the FP32 and FP64 instances, pair entries per
// chunk of the FP32 instances, entries per thread whose loads are issued together, and
// whether the tile's own records are prefetched into L1 ahead of the integration.
#ifndef DEM_TILED_BLOCKS32
#define DEM_TILED_BLOCKS32 3
#endif
#ifndef DEM_TILED_BLOCKS64
#define DEM_TILED_BLOCKS64 2
#endif
#ifndef DEM_TILE_CHUNK32
#define DEM_TILE_CHUNK32 (4 * DEM_TILE_THREADS)
#endif
#ifndef DEM_TILE_BATCH32
#define DEM_TILE_BATCH32 4
#endif
#ifndef DEM_TILED_PREFETCH
#define DEM_TILED_PREFETCH 1
#endif
constexpr int kTiledBlocks32 = DEM_TILED_BLOCKS32;
constexpr int kTiledBlocks64 = DEM_TILED_BLOCKS64;

template <bool FP32, bool EVAL>
struct TileSmem {
  static constexpr int kPairChunk = (FP32 && !EVAL) ? DEM_TILE_CHUNK32 : 2 * kTileThreads;  // pair entries per chunk
  static constexpr int kBondChunk = 2 * kTileThreads;               // bond entries per chunk (FP64 sums)
  static constexpr int kChunkMax = kPairChunk > kBondChunk ? kPairChunk : kBondChunk;
  using T = typename std::conditional<FP32, float, double>::type;
  int start[kTileThreads + 1];     // the tile's adjacency starts
  int owner[kChunkMax];            // local particle of each entry of the chunk
  unsigned char live[kChunkMax];   // entry contributes (touching pair / intact bond)
  unsigned char alive[kTileThreads];  // bit 0 alive; bit 1 its hand-off flag
  double4 p[kTileThreads];         // the tile's positions and radii
  union {
    struct { T f[3][kPairChunk]; T m[3][kPairChunk]; } pair;
    struct { double f[3][kBondChunk]; double m[3][kBondChunk]; } bond;
  } c;
  double g[EVAL ? kChunkMax : 1];  // evaluation pass: magnitudes of the contributions
};

// Entries per thread whose loads are issued together.
template <bool FP32>
struct TileBatch {
  static constexpr int value = FP32 ? DEM_TILE_BATCH32 : 2;
};

// Contact test of pair entry u of the chunk (adjacency entry en of group G, partner record
// pj).  Returns true when the entry needs its law evaluated; otherwise the entry contributes
// nothing and, on the p1 side of a friction pair, its history is cleared here.
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ bool tile_pair_test(const StepArgs& a, const DynDev& G, int u, int2 en, const double4& pj,
                                               long long step, const TileSmem<FP32, EVAL>& S) {
  const int o = S.owner[u];
  if (!S.alive[o]) return false;
  const bool isp1 = en.y < 0;
  const int k = en.y & kAdjIndex;
  bool clear = false, eval = false;
  // device bond hand-off: skipped while the bond that excluded it holds
  const bool held = handoff_held<FEAT>(a, G, en.y, (S.alive[o] & 2) != 0, step);
  if (held) {
    clear = true;
  } else {
    const double4 ps = S.p[o];
    const double4 pa = isp1 ? ps : pj, pb = isp1 ? pj : ps;
    const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
    const V D = x1 - x2;
    const double eq_dist = pa.w + pb.w;
    const bool touching = dot(D, D) < (eq_dist * eq_dist);  // the laws' contact test
    if (G.kind == 0) {
      eval = (FEAT & F_ELASTIC) != 0 && touching;
    } else if (ROT && (FEAT & F_FRIC) != 0) {
      eval = touching;
      clear = !touching;  // CRotFrictionInteraction::calcSimpleForces, no-contact branch
    }
  }
  if (clear && isp1 && !EVAL) {
    if (FP32) G.hist32_out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    else G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
  }
  return eval;
}

// Law of a touching pair entry u (adjacency entry en of group G, partner record pj): its
// contribution to the entry's own particle.  Returns whether it contributes.
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ bool tile_pair_law(const StepArgs& a, const ParticleBuf& in, const DynDev& G, int i0, int u,
                                              int2 en, const double4& pj, TileSmem<FP32, EVAL>& S) {
  using T = typename TileSmem<FP32, EVAL>::T;
  const int o = S.owner[u];
  const int j = en.x;
  const bool isp1 = en.y < 0;
  const int k = en.y & kAdjIndex;
  const double4 ps = S.p[o];
  const double4 pa = isp1 ? ps : pj, pb = isp1 ? pj : ps;
  const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
  const V D = x1 - x2;
  T f[3] = {T(0), T(0), T(0)}, m[3] = {T(0), T(0), T(0)};
  double gs = 0.0;
  bool live = false;
  if (G.kind == 0) {
    if constexpr ((FEAT & F_ELASTIC) != 0) {
      if constexpr (!FP32) {
        V F;
        if (law_elastic(elastic_k(G.k, G.scaling, pa.w, pb.w), x1, pa.w, x2, pb.w, F)) {
          if (isp1) F = -1.0 * F;
          f[0] = F.x; f[1] = F.y; f[2] = F.z;
          live = true;
        }
      } else {
        Vf F;
        if (law_elastic_f32(elastic_k(G.k, G.scaling, pa.w, pb.w), D, pa.w, pb.w, F)) {
          if (isp1) F = -F;
          f[0] = F.x; f[1] = F.y; f[2] = F.z;
          if (EVAL) gs = (double)norm(F);
          live = true;
        }
      }
    }
  } else {
    if constexpr (ROT && (FEAT & F_FRIC) != 0) {
      const int io = i0 + o;
      double keff, kseff;
      friction_k(G.k, G.ks, G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
      if constexpr (!FP32) {
        const double4 vo = ldg4(in.vm + io), wo = ldg4(in.wi + io);
        const double4 vj = ldg4(in.vm + j), wj = ldg4(in.wi + j);
        const double4 va = isp1 ? vo : vj, vb = isp1 ? vj : vo;
        const double4 wa = isp1 ? wo : wj, wb = isp1 ? wj : wo;
        const double4 h = ldg4(G.hist_in + k);
        FricOut r;
        law_friction(keff, kseff, G.mu_s, G.mu_d, G.dt, x1, pa.w, xyz(va), xyz(wa), x2, pb.w, xyz(vb), xyz(wb),
                     mk(h.x, h.y, h.z), (((int)h.w) & 1) != 0, r);
        // p1: -force + Ffric and M1; p2: force - Ffric and M2 (the exact negation of p1's force)
        const V F = isp1 ? (-1.0 * r.fn) + r.Ffric : r.fn + (-1.0 * r.Ffric);
        const V M = isp1 ? r.M1 : r.M2;
        f[0] = F.x; f[1] = F.y; f[2] = F.z;
        m[0] = M.x; m[1] = M.y; m[2] = M.z;
        if (isp1)
          G.hist_out[k] = make_double4(r.Ffric.x, r.Ffric.y, r.Ffric.z,
                                       (r.slipping ? 1.0 : 0.0) + (r.touching ? 2.0 : 0.0));
      } else {
        const float4 s0 = __ldg(in.vw + 2 * io), s1 = __ldg(in.vw + 2 * io + 1);
        const float4 r0 = __ldg(in.vw + 2 * j), r1 = __ldg(in.vw + 2 * j + 1);
        const Vf vo = mk(s0.x, s0.y, s0.z), wo = mk(s0.w, s1.x, s1.y);
        const Vf vj = mk(r0.x, r0.y, r0.z), wj = mk(r0.w, r1.x, r1.y);
        Vf hF;
        bool hs;
        if (EVAL) {  // evaluation pass of an FP64 run: its FP64 history
          const double4 h = ldg4(G.hist_in + k);
          hF = mk((float)h.x, (float)h.y, (float)h.z);
          hs = (((int)h.w) & 1) != 0;
        } else {
          const float4 h = __ldg(G.hist32_in + k);
          hF = mk(h.x, h.y, h.z);
          hs = (((int)h.w) & 1) != 0;
        }
        FricOutF r;
        law_friction_f32(keff, kseff, G.mu_s, G.mu_d, (float)G.dt, D, pa.w, pb.w, isp1 ? vo : vj, isp1 ? wo : wj,
                         isp1 ? vj : vo, isp1 ? wj : wo, hF, hs, r);
        const Vf F = isp1 ? (-r.fn) + r.Ffric : r.fn + (-r.Ffric);
        const Vf M = isp1 ? r.M1 : r.M2;
        f[0] = F.x; f[1] = F.y; f[2] = F.z;
        m[0] = M.x; m[1] = M.y; m[2] = M.z;
        if (EVAL) gs = (double)norm(r.fn) + (double)norm(r.Ffric);
        if (isp1 && !EVAL)
          G.hist32_out[k] = make_float4(r.Ffric.x, r.Ffric.y, r.Ffric.z,
                                        (r.slipping ? 1.f : 0.f) + (r.touching ? 2.f : 0.f));
      }
      live = true;
    }
  }
  if (live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      S.c.pair.f[c][u] = f[c];
      if (ROT) S.c.pair.m[c][u] = m[c];
    }
    if constexpr (EVAL) S.g[u] = gs;
  }
  return live;
}

// Entries [Eb, Eb + m) of group G: every thread takes entries u = t, t + kTileThreads, ...,
// issues the entry and partner loads of TileBatch of them at once and tests their contacts;
// the laws of the touching ones run afterwards, one at a time, from their inputs re-read
// (L1 hits), so that the batch stays in registers.
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ void tile_eval_pairs(const StepArgs& a, const ParticleBuf& in, const DynDev& G, int i0,
                                                int Eb, int m, long long step, TileSmem<FP32, EVAL>& S) {
  constexpr int kB = TileBatch<FP32>::value;
  for (int u0 = threadIdx.x; u0 < m; u0 += kB * kTileThreads) {
    int2 en[kB];
    double4 pj[kB];
#pragma unroll
    for (int b = 0; b < kB; ++b) {
      const int u = u0 + b * kTileThreads;
      en[b] = u < m ? __ldg(G.adj + Eb + u) : make_int2(-1, 0);
    }
    // under the device bond hand-off a pair is skipped while its excluding bond holds: its partner
    // record is not needed (in a bonded specimen that is most of the friction list)
    bool held[kB];
#pragma unroll
    for (int b = 0; b < kB; ++b) {
      const int u = u0 + b * kTileThreads;
      held[b] = en[b].x >= 0 && handoff_held<FEAT>(a, G, en[b].y, (S.alive[S.owner[u]] & 2) != 0, step);
    }
#pragma unroll
    for (int b = 0; b < kB; ++b)
      pj[b] = (en[b].x >= 0 && !held[b]) ? ldg4(in.pr + en[b].x) : make_double4(0.0, 0.0, 0.0, 0.0);
    unsigned todo = 0u;
#pragma unroll
    for (int b = 0; b < kB; ++b) {
      const int u = u0 + b * kTileThreads;
      if (u < m) {
        const bool ev = tile_pair_test<ROT, FEAT, FP32, EVAL>(a, G, u, en[b], pj[b], step, S);
        if (ev) todo |= 1u << b;
        else S.live[u] = 0;
      }
    }
    while (todo) {
      const int b = __ffs(todo) - 1;
      todo &= todo - 1u;
      const int u = u0 + b * kTileThreads;
      const int2 e = __ldg(G.adj + Eb + u);
      S.live[u] = tile_pair_law<ROT, FEAT, FP32, EVAL>(a, in, G, i0, u, e, ldg4(in.pr + e.x), S) ? 1 : 0;
    }
  }
}

// Bond entries [Eb, Eb + m) of group B (bond pass results): the force and moment on the
// entry's own particle.  A bond removed by an earlier update carries zero records.
template <bool ROT, bool FP32, bool EVAL>
__device__ __forceinline__ void tile_eval_bonds(const BondDev& B, int Eb, int m, long long step,
                                                TileSmem<FP32, EVAL>& S) {
  for (int u = threadIdx.x; u < m; u += kTileThreads) {
    const int2 en = __ldg(B.adj + Eb + u);
    const int k = en.y & 0x7fffffff;
    const bool live = S.alive[S.owner[u]];
    if (live) {
      const bool isp1 = en.y < 0;
      V F, M = mk(0.0, 0.0, 0.0);
      if constexpr (FP32 && !EVAL) {
        const float4* rf = B.bf32 + 4 * (size_t)k + (isp1 ? 0 : 2);
        const float4 a0 = __ldg(rf), a1 = __ldg(rf + 1);
        F = mk((double)a0.x, (double)a0.y, (double)a0.z);
        if (ROT) M = mk((double)a0.w, (double)a1.x, (double)a1.y);
      } else {
        const double4* r = B.bf + 3 * (size_t)k;
        const double4 f = ldg4(r);
        F = isp1 ? xyz(f) : -1.0 * xyz(f);
        if (ROT) M = xyz(ldg4(r + (isp1 ? 1 : 2)));
      }
      S.c.bond.f[0][u] = F.x;
      S.c.bond.f[1][u] = F.y;
      S.c.bond.f[2][u] = F.z;
      if (ROT) {
        S.c.bond.m[0][u] = M.x;
        S.c.bond.m[1][u] = M.y;
        S.c.bond.m[2][u] = M.z;
      }
      if constexpr (EVAL) S.g[u] = norm(F);
    }
    S.live[u] = live ? 1 : 0;
  }
}

// Pair-group and bond sums of the tile's particles [i0, i0 + np).  Every thread of the
// block calls this; thread t returns the sums of particle i0 + t.  Order per particle:
// the groups in order, each group's entries in adjacency order; FP32 pair contributions
// through the compensated sum, bond contributions in FP64 (as pair_sums does).
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ void tile_pair_sums(const StepArgs& a, const ParticleBuf& in, int i0, int np,
                                               long long step, TileSmem<FP32, EVAL>& S, V& Fp, V& Mp, double& Gs) {
  using Sm = TileSmem<FP32, EVAL>;
  const int t = threadIdx.x;
  Fp = mk(0.0, 0.0, 0.0);
  Mp = mk(0.0, 0.0, 0.0);
  Gs = 0.0;
  KSum3 Fk, Mk;
  Fk.zero();
  Mk.zero();
  if (np <= 0) return;  // uniform over the block: an empty specimen's single tile
  if constexpr ((FEAT & (F_ELASTIC | F_FRIC)) != 0) {
    for (int d = 0; d < a.ndyn; ++d) {
      const DynDev& G = a.dyn[d];
      if (d > 0) {  // group 0's starts were loaded with the tile's own records (tile_own)
        __syncthreads();  // the previous group's starts and owners are no longer read
        if (t < np) S.start[t] = __ldg(G.adj_start + i0 + t);
        if (t == 0) S.start[np] = __ldg(G.adj_start + i0 + np);
      }
      __syncthreads();
      const int E0 = S.start[0], cnt = S.start[np] - E0;
      const int my0 = t < np ? S.start[t] - E0 : 0, my1 = t < np ? S.start[t + 1] - E0 : 0;
      for (int c = 0; c < cnt; c += Sm::kPairChunk) {
        const int ce = min(cnt, c + Sm::kPairChunk);
        for (int q = max(my0, c); q < min(my1, ce); ++q) S.owner[q - c] = t;
        __syncthreads();
        tile_eval_pairs<ROT, FEAT, FP32, EVAL>(a, in, G, i0, E0 + c, ce - c, step, S);
        __syncthreads();
        for (int q = max(my0, c); q < min(my1, ce); ++q) {
          const int u = q - c;
          if (!S.live[u]) continue;
          if constexpr (FP32) {
            Fk.add(mk(S.c.pair.f[0][u], S.c.pair.f[1][u], S.c.pair.f[2][u]));
            if (ROT) Mk.add(mk(S.c.pair.m[0][u], S.c.pair.m[1][u], S.c.pair.m[2][u]));
          } else {
            Fp += mk((double)S.c.pair.f[0][u], (double)S.c.pair.f[1][u], (double)S.c.pair.f[2][u]);
            if (ROT) Mp += mk((double)S.c.pair.m[0][u], (double)S.c.pair.m[1][u], (double)S.c.pair.m[2][u]);
          }
          if constexpr (EVAL) Gs += S.g[u];
        }
        __syncthreads();  // contributions read before the next chunk overwrites them
      }
    }
  }
  if constexpr ((FEAT & F_BGATHER) != 0) {
    for (int d = 0; d < a.nbond; ++d) {
      const BondDev& B = a.bond[d];
      __syncthreads();
      if (t < np) S.start[t] = __ldg(B.adj_start + i0 + t);
      if (t == 0) S.start[np] = __ldg(B.adj_start + i0 + np);
      __syncthreads();
      const int E0 = S.start[0], cnt = S.start[np] - E0;
      const int my0 = t < np ? S.start[t] - E0 : 0, my1 = t < np ? S.start[t + 1] - E0 : 0;
      for (int c = 0; c < cnt; c += Sm::kBondChunk) {
        const int ce = min(cnt, c + Sm::kBondChunk);
        for (int q = max(my0, c); q < min(my1, ce); ++q) S.owner[q - c] = t;
        __syncthreads();
        tile_eval_bonds<ROT, FP32, EVAL>(B, E0 + c, ce - c, step, S);
        __syncthreads();
        for (int q = max(my0, c); q < min(my1, ce); ++q) {
          const int u = q - c;
          if (!S.live[u]) continue;
          Fp += mk(S.c.bond.f[0][u], S.c.bond.f[1][u], S.c.bond.f[2][u]);
          if (ROT) Mp += mk(S.c.bond.m[0][u], S.c.bond.m[1][u], S.c.bond.m[2][u]);
          if constexpr (EVAL) Gs += S.g[u];
        }
        __syncthreads();
      }
    }
  }
  if (FP32) {  // FP64-form sums (bonds) are added after the compensated FP32 pair sums
    Fp = Fk.value() + Fp;
    Mp = Mk.value() + Mp;
  }
}

// The tile's own loads: flags, position into shared memory, the records read after the
// pair phase into L1.
// The tile's own loads, all issued at once: flags and position into shared memory, the
// first pair group's adjacency starts (tile_pair_sums reads them from S.start), and the
// records read after the pair phase into L1.
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ void tile_own(const StepArgs& a, const ParticleBuf& in, int i0, int np, unsigned& pf,
                                         double4& p4, TileSmem<FP32, EVAL>& S) {
  const int t = threadIdx.x, i = i0 + t;
  const bool valid = t < np;
  constexpr bool kPairs = (FEAT & (F_ELASTIC | F_FRIC)) != 0;
  const bool starts = kPairs && a.ndyn > 0 && np > 0;
  pf = 0u;
  p4 = make_double4(0, 0, 0, 0);
  int st = 0, st_end = 0;
  if (valid) {
    pf = __ldg(a.P.pflags + i);
    p4 = ldg4(in.pr + i);
    if (starts) st = __ldg(a.dyn[0].adj_start + i);
    if (DEM_TILED_PREFETCH) {
      prefetch_l1(in.vm + i);
      if (ROT) { prefetch_l1(in.wi + i); prefetch_l1(in.qq + i); }
      if (FP32 && ROT) prefetch_l1(in.vw + 2 * i);
    }
  }
  if (starts && t == 0) st_end = __ldg(a.dyn[0].adj_start + i0 + np);
  __syncthreads();  // the previous tile's pair phase has finished with S.p / S.alive / S.start
  S.p[t] = p4;
  // bit 0 alive, bit 1 the hand-off flag of a live particle (handoff_held)
  S.alive[t] = (valid && (pf & PF_ALIVE)) ? (handoff_flag<FEAT>(a, i) ? 3 : 1) : 0;
  if (starts) {
    if (valid) S.start[t] = st;
    if (t == 0) S.start[np] = st_end;
  }
}

template <bool ROT, int FEAT, bool FP32, bool EVAL>
__global__ void __launch_bounds__(kTileThreads, FP32 ? kTiledBlocks32 : kTiledBlocks64) k_step_tiled(const StepArgs a) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  __shared__ TileSmem<FP32, EVAL> S;
  if (!EVAL && *a.stop) return;  // an earlier step of this chunk asked the host to intervene
  const long long step = *a.step_counter + 1;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const ParticleBuf in = a.P.buf[a.cur];
  const ParticleBuf out = a.P.buf[a.cur ^ 1];
  for (int k = threadIdx.x; k < kStepWarps * kMaxWalls * 3; k += kTileThreads) (&s_red[0][0][0])[k] = 0.0;
  const int ntiles = step_tiles(a.P.n, kTiled);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i0 = tile * kTileThreads;
    const int np = min(kTileThreads, a.P.n - i0);
    const int i = i0 + threadIdx.x;
    const bool valid = (int)threadIdx.x < np;
    unsigned pf;
    double4 p4;
    tile_own<ROT, FEAT, FP32, EVAL>(a, in, i0, np, pf, p4, S);
    const bool alive = valid && (pf & PF_ALIVE);
    V Fp, Mp;
    double gross;
    tile_pair_sums<ROT, FEAT, FP32, EVAL>(a, in, i0, max(np, 0), step, S, Fp, Mp, gross);
    finish_particle<ROT, 1, FP32, EVAL>(a, step, in, out, i, 0, wlane, warp, pf, alive, p4, make_double4(1, 0, 0, 0),
                                        false, Fp, Mp, s_red);
    // evaluation pass: the particle's contact-force scale beside its force (w of the record)
    if (EVAL && alive) reinterpret_cast<double*>(a.P.force_eval + i)[3] = gross;
  }
  if (EVAL) return;
  step_epilogue(a, step, wlane, warp, s_red, &s_last);
}

template <bool R, int FEAT, bool FP32, bool EVAL>
inline void launch_tiled(const StepArgs& a, cudaStream_t s) {
  const int tiles = step_blocks(a.P.n, kTiled);
  const int wave = one_wave(k_step_tiled<R, FEAT, FP32, EVAL>, kTileThreads);
  k_step_tiled<R, FEAT, FP32, EVAL><<<tiles < wave ? tiles : wave, kTileThreads, 0, s>>>(a);
}

template <bool R, int FEAT, bool FP32, bool EVAL>
inline void launch_step_tpp(const StepArgs& a, int tpp, cudaStream_t s) {
  if (tpp == kTiled) {
    if constexpr (TiledSupported<FEAT>::value) return launch_tiled<R, FEAT, FP32, EVAL>(a, s);
    tpp = 1;
  }
  if (tpp == kWarpCoop) {
    if constexpr (WarpCoopSupported<FEAT>::value) return launch_fused<R, kWarpCoop, FEAT, FP32, EVAL>(a, s);
    tpp = 1;
  }
  switch (tpp) {
    case 1: launch_fused<R, 1, FEAT, FP32, EVAL>(a, s); break;
    case 2: launch_fused<R, 2, FEAT, FP32, EVAL>(a, s); break;
    case 4: launch_fused<R, 4, FEAT, FP32, EVAL>(a, s); break;
    default: launch_fused<R, 8, FEAT, FP32, EVAL>(a, s); break;
  }
}

}  // namespace dem
