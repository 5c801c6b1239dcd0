// FP32-force instances of the step kernel (see dem_step.cuh): pair forces in
// FP32 with Kahan-compensated accumulation, positions / contact detection /
// overlap / integration in FP64.  Built with FMA contraction (the FP32 form is
// checked against FP64 at a stated relative tolerance, not bit for bit).
#include "dem_kernels.h"
#include "dem_tiled.cuh"

namespace dem {

void launch_step_fp32(const StepArgs& a, bool rot, int tpp, bool eval, bool split, cudaStream_t s) {
  bool el = false, fr = false;
  for (int d = 0; d < a.ndyn; ++d) (a.dyn[d].kind == 0 ? el : fr) = true;
  const bool bd = a.nbond > 0;
  const bool gather = bd && a.bond[0].bf;  // bonds evaluated once by the bond pass
  if (gather) launch_bond_pass_f64(a, eval, s);  // FP64, uncontracted: the FP64 form's bond forces
  if (split && !eval) {
    if (!rot) return launch_split_tpp<false, F_ELASTIC, true>(a, tpp, s);
    if (!bd && fr && !el) return launch_split_tpp<true, F_FRIC, true>(a, tpp, s);
    if (!bd && !fr) return launch_split_tpp<true, F_ELASTIC, true>(a, tpp, s);
    if (gather) return launch_split_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, true>(a, tpp, s);
    return launch_split_tpp<true, F_ELASTIC | F_FRIC | F_BOND, true>(a, tpp, s);
  }
  if (eval) {
    if (!rot) return launch_step_tpp<false, F_ELASTIC, true, true>(a, tpp, s);
    if (!bd && fr && !el) return launch_step_tpp<true, F_FRIC, true, true>(a, tpp, s);
    if (!bd && !fr) return launch_step_tpp<true, F_ELASTIC, true, true>(a, tpp, s);
    if (gather) return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, true, true>(a, tpp, s);
    return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BOND, true, true>(a, tpp, s);
  }
  if (!rot) return launch_step_tpp<false, F_ELASTIC, true, false>(a, tpp, s);
  if (!bd && fr && !el) return launch_step_tpp<true, F_FRIC, true, false>(a, tpp, s);
  if (!bd && !fr) return launch_step_tpp<true, F_ELASTIC, true, false>(a, tpp, s);
  if (gather && !el) return launch_step_tpp<true, F_FRIC | F_BGATHER, true, false>(a, tpp, s);
  if (gather) return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BGATHER, true, false>(a, tpp, s);
  return launch_step_tpp<true, F_ELASTIC | F_FRIC | F_BOND, true, false>(a, tpp, s);
}

}  // namespace dem
