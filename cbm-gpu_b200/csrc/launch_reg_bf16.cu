// Register-gather forward kernel instantiations, BF16 X.
#include "launch.cuh"

namespace cbm {
int launch_fwd_bf16(cbm_plan* P, const FwdArgs& a, int32_t ydt, bool vec, int vpl, bool wide, cudaStream_t st) {
  if (ydt == CBM_F32 && wide && vpl == 1) {
    return vec ? launch_fwd_t<__nv_bfloat16, float, 1, 8, false, true>(P, a, st)
               : launch_fwd_t<__nv_bfloat16, float, 1, 1, false, true>(P, a, st);
  }
  if (ydt == CBM_F32) {
    return vec ? launch_fwd_v<__nv_bfloat16, float, 8>(P, a, vpl, st)
               : launch_fwd_v<__nv_bfloat16, float, 1>(P, a, vpl, st);
  }
  return vec ? launch_fwd_v<__nv_bfloat16, __nv_bfloat16, 8>(P, a, vpl, st)
             : launch_fwd_v<__nv_bfloat16, __nv_bfloat16, 1>(P, a, vpl, st);
}
}  // namespace cbm
