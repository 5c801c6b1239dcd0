// Allocation-free wall reactions: dem_wall_reactions_noalloc (include/esys_dem.h).
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured (allocation is not a capturable operation), hosts that give
// the library only memory from their own pool, and real-time loops that forbid
// allocation after start-up.  This entry point computes per-wall reaction forces
// (the sum over the given particles of their elastic wall contact forces) and keeps
// its block-partial sums in a fixed device array instead of memory it allocates.
// Every given particle counts, wherever it lies; the step kernel's reaction
// (CWall::m_force) counts only the wall's candidates (particles within one grid
// spacing of the plane, in the grid interior), so the two agree when the given
// particles are those candidates, e.g. all particles of a closed box.
//
// The array is a file-scope __device__ object: every GPU that loads the library
// holds its 111 KiB (113,672 bytes) until the process exits, and every call on that GPU shares
// it, so two calls that run at the same time on the same GPU (different
// streams, overlapping) race and give wrong sums.
#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/esys_dem.h"
#include "dem_laws.cuh"

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxBlocks = 592;    // 148 SMs x 4: the grid strides over the particles
constexpr int kNaMaxWalls = 8;
constexpr int kNaMaxParticles = 1 << 24;

// Block partial sums [block][wall][xyz] followed by the last-block counter.
struct NoAllocScratch {
  double partial[kNaMaxBlocks][kNaMaxWalls][3];
  unsigned counter;
};
static_assert(sizeof(NoAllocScratch) == 113672, "the documented size of the scratch array");
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Per-particle elastic wall forces (CElasticWallInteraction::calcForces,
// Model/EWallInteraction.hpp:42-78) summed per wall in a fixed order: thread
// stride, warp shuffle, warps, then blocks in index order in the last block.
__global__ void __launch_bounds__(kNaThreads) k_wall_reactions_noalloc(int n, const double4* __restrict__ pr,
                                                                      int nwall, const double* __restrict__ walls,
                                                                      double* __restrict__ out,
                                                                      NoAllocScratch* scratch) {
  __shared__ double s_red[kNaThreads / 32][kNaMaxWalls][3];
  __shared__ bool s_last;
  const int wl = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (int w = 0; w < nwall; ++w) {
    const double* W = walls + 7 * w;
    const dem::V o = dem::mk(W[0], W[1], W[2]), nrm = dem::mk(W[3], W[4], W[5]);
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const double4 p = pr[i];
      dem::V f;
      if (dem::law_wall(W[6], o, nrm, dem::mk(p.x, p.y, p.z), p.w, f)) { cx += f.x; cy += f.y; cz += f.z; }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      cx += __shfl_down_sync(0xffffffffu, cx, s);
      cy += __shfl_down_sync(0xffffffffu, cy, s);
      cz += __shfl_down_sync(0xffffffffu, cz, s);
    }
    if (wl == 0) { s_red[wp][w][0] = cx; s_red[wp][w][1] = cy; s_red[wp][w][2] = cz; }
  }
  __syncthreads();
  if (threadIdx.x < 3 * nwall) {
    const int w = threadIdx.x / 3, c = threadIdx.x % 3;
    double acc = 0.0;
    for (int k = 0; k < kNaThreads / 32; ++k) acc += s_red[k][w][c];
    scratch->partial[blockIdx.x][w][c] = acc;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicInc(&scratch->counter, gridDim.x - 1) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < 3 * nwall) {
    const int w = threadIdx.x / 3, c = threadIdx.x % 3;
    double acc = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) acc += __ldcg(&scratch->partial[b][w][c]);
    out[3 * w + c] = acc;
  }
}

// Device address of the scratch array, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

extern "C" int dem_wall_reactions_noalloc(int n, const double* particles, int nwall, const double* walls,
                                          double* reactions, void* stream) {
  if (n < 0 || n > kNaMaxParticles) return DEM_ERR_ARG;
  if (nwall < 1 || nwall > kNaMaxWalls) return DEM_ERR_ARG;
  if ((n > 0 && !particles) || !walls || !reactions) return DEM_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(particles) % 16 != 0) return DEM_ERR_ARG;  // double4 rows
  if (reinterpret_cast<uintptr_t>(walls) % 8 != 0 || reinterpret_cast<uintptr_t>(reactions) % 8 != 0)
    return DEM_ERR_ARG;  // doubles
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DEM_ERR_CUDA;
  NoAllocScratch* scratch = nullptr;
  {
    // Set-up on the first call on this device (the device current at the call):
    // the host needs the scratch array's device address.
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return DEM_ERR_CUDA;
      g_scratch_ptr[dev] = static_cast<NoAllocScratch*>(ptr);
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The counter must start at zero; the partials are fully rewritten by every call.
  if (cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned), s) != cudaSuccess) return DEM_ERR_CUDA;
  int blocks = (n + kNaThreads - 1) / kNaThreads;
  blocks = blocks < 1 ? 1 : (blocks > kNaMaxBlocks ? kNaMaxBlocks : blocks);
  k_wall_reactions_noalloc<<<blocks, kNaThreads, 0, s>>>(n, reinterpret_cast<const double4*>(particles), nwall,
                                                          walls, reactions, scratch);
  return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}
