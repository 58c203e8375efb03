// Staged forward kernel instantiations, BF16 X, FP32 Y.
#include "launch.cuh"

namespace cbm {
int launch_staged_bf16_f32(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st) {
  return launch_staged_any<__nv_bfloat16, float>(P, a, team, vpl, st);
}
}  // namespace cbm
