// Reverse-propagation (adjoint) kernel instantiations.
#include "launch.cuh"

namespace cbm {
template <typename GT, int V>
int launch_rev_v(cbm_plan* P, const RevArgs& a, int vpl, cudaStream_t st) {
  switch (vpl) {
    case 1: return launch_rev_t<GT, 1, V>(P, a, st);
    case 2: return launch_rev_t<GT, 2, V>(P, a, st);
    case 4: return launch_rev_t<GT, 4, V>(P, a, st);
    default: return launch_rev_t<GT, 8, V>(P, a, st);
  }
}

int launch_rev(cbm_plan* P, const RevArgs& a, int32_t gdt, bool vec, int vpl, cudaStream_t st) {
  if (gdt == CBM_F32) return vec ? launch_rev_v<float, 4>(P, a, vpl, st) : launch_rev_v<float, 1>(P, a, vpl, st);
  return vec ? launch_rev_v<__nv_bfloat16, 8>(P, a, vpl, st) : launch_rev_v<__nv_bfloat16, 1>(P, a, vpl, st);
}
}  // namespace cbm
