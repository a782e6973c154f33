// dg_k_x2_small.cu — instances of the packed two-shot kernels for 2, 4, 6 and 8 stored shots
// (element-major and plane-major layouts, plain and Kahan).
#include "dg_kernels.cuh"

namespace dg {

HalfPair<X2Fn> kernels_packed_small(int S, bool kahan, bool pm) {
#define DG_X2(SS, KH, PM) \
  if (S == SS && kahan == KH && pm == PM) return {k_velocity_x2<SS, KH, PM>, k_stress_x2<SS, KH, PM>};
#define DG_X2ALL(SS) DG_X2(SS, false, false) DG_X2(SS, true, false) DG_X2(SS, false, true) DG_X2(SS, true, true)
  DG_X2ALL(2) DG_X2ALL(4) DG_X2ALL(6) DG_X2ALL(8)
#undef DG_X2ALL
#undef DG_X2
  return {};
}

}  // namespace dg
