// Register-gather forward kernel instantiations: FP32 X, the compensated
// (precision-form) BF16 kernels, and the second pass of two-pass products.
#include "launch.cuh"

namespace cbm {
int launch_fwd_f32(cbm_plan* P, const FwdArgs& a, bool vec, int vpl, cudaStream_t st) {
  return vec ? launch_fwd_v<float, float, 4>(P, a, vpl, st) : launch_fwd_v<float, float, 1>(P, a, vpl, st);
}

int launch_fwd_comp(cbm_plan* P, const FwdArgs& a, int32_t ydt, bool vec, int vpl, cudaStream_t st) {
  if (ydt == CBM_F32) {
    return vec ? launch_fwd_v<__nv_bfloat16, float, 8, true>(P, a, vpl, st)
               : launch_fwd_v<__nv_bfloat16, float, 1, true>(P, a, vpl, st);
  }
  return vec ? launch_fwd_v<__nv_bfloat16, __nv_bfloat16, 8, true>(P, a, vpl, st)
             : launch_fwd_v<__nv_bfloat16, __nv_bfloat16, 1, true>(P, a, vpl, st);
}

int launch_prop(cbm_plan* P, const PropArgs& a, bool vec, int vpl, cudaStream_t st) {
  if (!vec) return vpl <= 1 ? launch_prop_t<1, 1>(P, a, st) : launch_prop_t<4, 1>(P, a, st);
  switch (vpl) {
    case 1: return launch_prop_t<1, 4>(P, a, st);
    case 2: return launch_prop_t<2, 4>(P, a, st);
    case 4: return launch_prop_t<4, 4>(P, a, st);
    default: return launch_prop_t<8, 4>(P, a, st);
  }
}
}  // namespace cbm
