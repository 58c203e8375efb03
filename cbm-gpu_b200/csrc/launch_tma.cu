// TMA (tile::gather4) forward kernel instantiations, all operand type pairs.
#include "launch.cuh"

namespace cbm {
int launch_tma(cbm_plan* P, const FwdArgs& a, int32_t xdt, int32_t ydt, int team, int vpl, const CUtensorMap& map,
               cudaStream_t st) {
  if (xdt == CBM_F32) return launch_tma_any<float, float>(P, a, team, vpl, map, st);
  if (ydt == CBM_F32) return launch_tma_any<__nv_bfloat16, float>(P, a, team, vpl, map, st);
  return launch_tma_any<__nv_bfloat16, __nv_bfloat16>(P, a, team, vpl, map, st);
}
}  // namespace cbm
