// Staged forward kernel instantiations, BF16 X and Y.
#include "launch.cuh"

namespace cbm {
int launch_staged_bf16_bf16(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st) {
  return launch_staged_any<__nv_bfloat16, __nv_bfloat16>(P, a, team, vpl, st);
}
}  // namespace cbm
