// Staged forward kernel instantiations, FP32 X and Y.
#include "launch.cuh"

namespace cbm {
int launch_staged_f32(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st) {
  return launch_staged_any<float, float>(P, a, team, vpl, st);
}
}  // namespace cbm
