// Batched ensemble step: many independent specimens (each one simulated worker
// with its own particles, interaction groups, walls and step counter) advance
// together, one launch per timestep for all of them.
//
// The launch is a persistent one-wave grid over the concatenated particle tiles
// of every specimen.  A tile maps to its specimen through a prefix table of tile
// counts; the specimen's step arguments (the same StepArgs its own k_step
// launch would get, for both buffer parities) are read from a device table, so
// a captured graph of launches stays valid while the table's contents change.
// Per tile the work is exactly k_step's per-particle work (pair_sums +
// finish_particle), hence per-particle results equal a specimen run alone.  The
// wall reactions are reduced per tile; the last tile of a specimen to finish
// (counted on the specimen's own counter) completes that specimen's step: wall
// totals, wall loaders, its step counter and its stop word.  A specimen whose
// stop word is set, or which has reached its target step, skips the launch.
#pragma once
#include "dem_kernels.h"
#include "dem_step.cuh"
#include "dem_tiled.cuh"

namespace dem {

__device__ __forceinline__ int batch_specimen(const BatchArgs& B, int tile) {
  int lo = 0, hi = B.nspec;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(B.tile_start + mid) <= tile) lo = mid; else hi = mid;
  }
  return lo;
}

// Per-tile wall partials, then the last tile of the specimen finishes its step
// (the same fixed-order reduction as step_epilogue, over the specimen's tiles).
__device__ __forceinline__ void batch_tile_epilogue(const StepArgs& a, long long step, int ltile, int ntiles,
                                                    int wlane, int warp, double (*s_red)[kMaxWalls][3],
                                                    bool* s_last) {
  if (!block_partials(a, ltile, ntiles, a.block_counter, s_red, s_last)) return;
  launch_tail(a, step, ntiles, wlane, warp);
}

template <bool ROT, int TPP, int FEAT, bool FP32>
__global__ void __launch_bounds__(kStepThreads, (FEAT & F_BOND) ? 1 : ((FEAT & F_BGATHER) ? 4 : (FP32 ? kFp32Blocks : 2)))
    k_step_batch(const BatchArgs B) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  const int lane = threadIdx.x % TPP;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int tile = blockIdx.x; tile < B.total_tiles; tile += gridDim.x) {
    const int sp = batch_specimen(B, tile);
    const StepArgs& a0 = B.args[2 * sp];
    // The specimen's counter and stop word change only in its own last tile, after every
    // tile of this launch has read them: the decision below is uniform over its tiles.
    const long long done = *(volatile long long*)a0.step_counter;
    if (*(volatile int*)a0.stop || done >= __ldg(B.target + sp)) continue;
    const int cur = (int)((done - __ldg(B.base_t + sp) + __ldg(B.base_cur + sp)) & 1);
    const StepArgs& a = B.args[2 * sp + cur];
    const long long step = done + 1;
    const int t0 = __ldg(B.tile_start + sp);
    const int ltile = tile - t0, ntiles = __ldg(B.tile_start + sp + 1) - t0;
    const ParticleBuf in = a.P.buf[a.cur];
    const ParticleBuf out = a.P.buf[a.cur ^ 1];
    __syncthreads();  // the previous tile's epilogue has finished with s_red
    for (int k = threadIdx.x; k < kStepWarps * kMaxWalls * 3; k += kStepThreads) (&s_red[0][0][0])[k] = 0.0;
    __syncthreads();
    const int i = (ltile * kStepThreads + threadIdx.x) / TPP;
    const bool valid = i < a.P.n;
    unsigned pf = 0u;
    double4 p4 = make_double4(0, 0, 0, 0), q4 = make_double4(1, 0, 0, 0);
    if (valid) {
      pf = __ldg(a.P.pflags + i);
      p4 = ldg4(in.pr + i);
      if (lane == 0) {
        prefetch_l1(in.vm + i);
        if (ROT) { prefetch_l1(in.wi + i); prefetch_l1(in.qq + i); }
        if (FP32 && ROT) prefetch_l1(in.vw + 2 * i);
      }
      if (ROT && (FEAT & F_BOND)) q4 = ldg4(in.qq + i);
    }
    const bool alive = valid && (pf & PF_ALIVE);
    V Fp, Mp;
    pair_sums<ROT, TPP, FEAT, FP32, false>(a, in, i, lane, alive, step, p4, q4, Fp, Mp);
    finish_particle<ROT, TPP, FP32, false>(a, step, in, out, i, lane, wlane, warp, pf, alive, p4, q4,
                                           ROT && (FEAT & F_BOND), Fp, Mp, s_red);
    batch_tile_epilogue(a, step, ltile, ntiles, wlane, warp, s_red, &s_last);
  }
}

// Tiled form of k_step_batch (dem_tiled.cuh): the tile's pair and bond entries are
// evaluated by the whole block, then each particle adds its entries in adjacency order.
template <bool ROT, int FEAT, bool FP32>
__global__ void __launch_bounds__(kTileThreads, FP32 ? kTiledBlocks32 : kTiledBlocks64) k_step_batch_tiled(const BatchArgs B) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  __shared__ TileSmem<FP32, false> S;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int tile = blockIdx.x; tile < B.total_tiles; tile += gridDim.x) {
    const int sp = batch_specimen(B, tile);
    const StepArgs& a0 = B.args[2 * sp];
    // The specimen's counter and stop word change only in its own last tile, after every
    // tile of this launch has read them: the decision below is uniform over its tiles.
    const long long done = *(volatile long long*)a0.step_counter;
    if (*(volatile int*)a0.stop || done >= __ldg(B.target + sp)) continue;
    const int cur = (int)((done - __ldg(B.base_t + sp) + __ldg(B.base_cur + sp)) & 1);
    const StepArgs& a = B.args[2 * sp + cur];
    const long long step = done + 1;
    const int t0 = __ldg(B.tile_start + sp);
    const int ltile = tile - t0, ntiles = __ldg(B.tile_start + sp + 1) - t0;
    const ParticleBuf in = a.P.buf[a.cur];
    const ParticleBuf out = a.P.buf[a.cur ^ 1];
    __syncthreads();  // the previous tile's epilogue has finished with s_red
    for (int k = threadIdx.x; k < kStepWarps * kMaxWalls * 3; k += kTileThreads) (&s_red[0][0][0])[k] = 0.0;
    const int i0 = ltile * kTileThreads;
    const int np = max(0, min(kTileThreads, a.P.n - i0));
    const int i = i0 + threadIdx.x;
    const bool valid = (int)threadIdx.x < np;
    unsigned pf;
    double4 p4;
    tile_own<ROT, FEAT, FP32, false>(a, in, i0, np, pf, p4, S);
    const bool alive = valid && (pf & PF_ALIVE);
    V Fp, Mp;
    double gross;
    tile_pair_sums<ROT, FEAT, FP32, false>(a, in, i0, np, step, S, Fp, Mp, gross);
    finish_particle<ROT, 1, FP32, false>(a, step, in, out, i, 0, wlane, warp, pf, alive, p4, make_double4(1, 0, 0, 0), false,
                                         Fp, Mp, s_red);
    batch_tile_epilogue(a, step, ltile, ntiles, wlane, warp, s_red, &s_last);
  }
}

// Batched bond pass: tiles of kBondPassThreads bonds over (specimen, bond group) items; an
// item without bonds has no tiles, so the last item whose first tile is <= tile owns it.
template <bool FP32>
__global__ void __launch_bounds__(kBondPassThreads, 4) k_bond_pass_batch(const BatchArgs B) {
  const int items = B.nspec * kMaxBond;
  for (int tile = blockIdx.x; tile < B.total_btiles; tile += gridDim.x) {
    int lo = 0, hi = items;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(B.btile_start + mid) <= tile) lo = mid; else hi = mid;
    }
    const int sp = lo / kMaxBond, d = lo % kMaxBond;
    const StepArgs& a0 = B.args[2 * sp];
    const long long done = *(volatile long long*)a0.step_counter;
    if (*(volatile int*)a0.stop || done >= __ldg(B.target + sp)) continue;
    const int cur = (int)((done - __ldg(B.base_t + sp) + __ldg(B.base_cur + sp)) & 1);
    const StepArgs& a = B.args[2 * sp + cur];
    const int k = (tile - __ldg(B.btile_start + lo)) * kBondPassThreads + threadIdx.x;
    if (k < a.bond[d].nb_launch) bond_pass_one<false>(a, a.bond[d], k, done + 1);
  }
}

template <bool FP32>
inline void launch_bond_pass_batch(const BatchArgs& B, cudaStream_t s) {
  if (B.total_btiles <= 0) return;
  static int wave = 0;  // per translation unit: one instance each
  if (!wave) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bond_pass_batch<FP32>, kBondPassThreads, 0);
    wave = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
  }
  const int grid = B.total_btiles < wave ? B.total_btiles : wave;
  k_bond_pass_batch<FP32><<<grid, kBondPassThreads, 0, s>>>(B);
}

template <bool R, int T, int FEAT, bool FP32>
inline void launch_batch_fixed(const BatchArgs& B, cudaStream_t s) {
  const int wave = one_wave(k_step_batch<R, T, FEAT, FP32>);
  const int grid = B.total_tiles < wave ? B.total_tiles : wave;
  if (grid > 0) k_step_batch<R, T, FEAT, FP32><<<grid, kStepThreads, 0, s>>>(B);
}

template <bool R, int FEAT, bool FP32>
inline void launch_batch_tiled(const BatchArgs& B, cudaStream_t s) {
  const int wave = one_wave(k_step_batch_tiled<R, FEAT, FP32>, kTileThreads);
  const int grid = B.total_tiles < wave ? B.total_tiles : wave;
  if (grid > 0) k_step_batch_tiled<R, FEAT, FP32><<<grid, kTileThreads, 0, s>>>(B);
}

template <bool R, int FEAT, bool FP32>
inline void launch_batch_tpp(const BatchArgs& B, int tpp, cudaStream_t s) {
  if (tpp == kTiled) {
    if constexpr (TiledSupported<FEAT>::value) return launch_batch_tiled<R, FEAT, FP32>(B, s);
    tpp = 1;
  }
  switch (tpp) {
    case 1: launch_batch_fixed<R, 1, FEAT, FP32>(B, s); break;
    case 2: launch_batch_fixed<R, 2, FEAT, FP32>(B, s); break;
    case 4: launch_batch_fixed<R, 4, FEAT, FP32>(B, s); break;
    default: launch_batch_fixed<R, 8, FEAT, FP32>(B, s); break;
  }
}

// Instances: non-rotational elastic; rotational friction, friction + bonds, and the general one.
template <bool FP32>
inline void launch_batch_any(const BatchArgs& B, bool rot, bool el, bool fr, bool bd, bool gather, int tpp,
                             cudaStream_t s) {
  if (!rot) return launch_batch_tpp<false, F_ELASTIC, FP32>(B, tpp, s);
  if (!bd && fr && !el) return launch_batch_tpp<true, F_FRIC, FP32>(B, tpp, s);
  if (gather) {
    launch_batch_bond_pass(B, s);  // FP64, uncontracted (dem_batch.cu), for both precision forms
    if (!el) return launch_batch_tpp<true, F_FRIC | F_BGATHER, FP32>(B, tpp, s);
    return launch_batch_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, FP32>(B, tpp, s);
  }
  if (bd && !el) return launch_batch_tpp<true, F_FRIC | F_BOND, FP32>(B, tpp, s);
  return launch_batch_tpp<true, F_ELASTIC | F_FRIC | F_BOND, FP32>(B, tpp, s);
}

}  // namespace dem
