// FP64 instances of the batched ensemble step (built with --fmad=false, like the
// single-specimen FP64 step) and the ensemble's small control kernels.
#include "dem_batch.cuh"
#include "dem_kernels.h"

namespace dem {

void launch_batch_step(const BatchArgs& B, bool rot, bool el, bool fr, bool bd, bool gather, int tpp,
                       cudaStream_t s) {
  launch_batch_any<false>(B, rot, el, fr, bd, gather, tpp, s);
}

void launch_batch_bond_pass(const BatchArgs& B, cudaStream_t s) { launch_bond_pass_batch<false>(B, s); }

// Clear every specimen's control and stop words before a chunk of steps.
__global__ void k_batch_reset(const StepArgs* args, int nspec) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nspec) return;
  *args[2 * k].ctrl = 0;
  *args[2 * k].stop = 0;
}

// Gather every specimen's step counter and control word into two arrays (one copy to the host).
__global__ void k_batch_status(const StepArgs* args, int nspec, long long* t, int* ctrl) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nspec) return;
  t[k] = *args[2 * k].step_counter;
  ctrl[k] = *args[2 * k].ctrl;
}

// FP32 shadow records (vw) of every specimen's input buffer: blockIdx.y is the specimen.
__global__ void k_batch_sync_vw(const StepArgs* args, const int* base_cur) {
  const int sp = blockIdx.y;
  const StepArgs& a = args[2 * sp + base_cur[sp]];
  const ParticleBuf b = a.P.buf[a.cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.P.n; i += gridDim.x * blockDim.x) {
    const double4 v = b.vm[i], w = b.wi[i];
    b.vw[2 * i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)w.x);
    b.vw[2 * i + 1] = make_float4((float)w.y, (float)w.z, 0.f, 0.f);
  }
}

void launch_batch_reset(const StepArgs* args, int nspec, cudaStream_t s) {
  if (nspec > 0) k_batch_reset<<<(nspec + 127) / 128, 128, 0, s>>>(args, nspec);
}
void launch_batch_status(const StepArgs* args, int nspec, long long* t, int* ctrl, cudaStream_t s) {
  if (nspec > 0) k_batch_status<<<(nspec + 127) / 128, 128, 0, s>>>(args, nspec, t, ctrl);
}
void launch_batch_sync_vw(const StepArgs* args, const int* base_cur, int nspec, cudaStream_t s) {
  if (nspec > 0) k_batch_sync_vw<<<dim3(16, nspec), 256, 0, s>>>(args, base_cur);
}

}  // namespace dem
