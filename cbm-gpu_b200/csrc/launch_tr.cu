// Transposed-gather (adjoint) kernel instantiations.
#include "launch.cuh"

namespace cbm {
// Rows narrower than a warp (teams of 1-16 lanes, one vector per lane) take
// the split kernel: the warp's lane groups share one column's entries.
constexpr bool kTrSplitNarrow = true;

template <typename GT, typename DT, int V>
int launch_tr_v(cbm_plan* P, const TrArgs& a, int vpl, cudaStream_t st) {
  if (kTrSplitNarrow && vpl == 1 && a.team < 32) return launch_tr_t<GT, DT, 1, V, true>(P, a, st);
  switch (vpl) {
    case 1: return launch_tr_t<GT, DT, 1, V>(P, a, st);
    case 2: return launch_tr_t<GT, DT, 2, V>(P, a, st);
    case 4: return launch_tr_t<GT, DT, 4, V>(P, a, st);
    default: return launch_tr_t<GT, DT, 8, V>(P, a, st);
  }
}

int launch_tr(cbm_plan* P, const TrArgs& a, int32_t gdt, int32_t ddt, bool vec, int vpl, cudaStream_t st) {
  if (gdt == CBM_F32) {
    return vec ? launch_tr_v<float, float, 4>(P, a, vpl, st) : launch_tr_v<float, float, 1>(P, a, vpl, st);
  }
  if (ddt == CBM_F32) {
    return vec ? launch_tr_v<__nv_bfloat16, float, 8>(P, a, vpl, st)
               : launch_tr_v<__nv_bfloat16, float, 1>(P, a, vpl, st);
  }
  return vec ? launch_tr_v<__nv_bfloat16, __nv_bfloat16, 8>(P, a, vpl, st)
             : launch_tr_v<__nv_bfloat16, __nv_bfloat16, 1>(P, a, vpl, st);
}
}  // namespace cbm
