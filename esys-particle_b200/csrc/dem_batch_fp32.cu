// FP32-force instances of the batched ensemble step (built with FMA contraction on,
// like the single-specimen FP32 step in dem_step_fp32.cu).
#include "dem_batch.cuh"
#include "dem_kernels.h"

namespace dem {

void launch_batch_step_fp32(const BatchArgs& B, bool rot, bool el, bool fr, bool bd, bool gather, int tpp,
                       cudaStream_t s) {
  launch_batch_any<true>(B, rot, el, fr, bd, gather, tpp, s);
}

}  // namespace dem
