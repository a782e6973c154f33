// dg_k_x2_mid.cu — instances of the packed two-shot kernels for 10, 12, 14 and 16 stored shots
// (element-major and plane-major layouts, plain and Kahan).
#include "dg_kernels.cuh"

namespace dg {

HalfPair<X2Fn> kernels_packed_mid(int S, bool kahan, bool pm) {
#define DG_X2(SS, KH, PM) \
  if (S == SS && kahan == KH && pm == PM) return {k_velocity_x2<SS, KH, PM>, k_stress_x2<SS, KH, PM>};
#define DG_X2ALL(SS) DG_X2(SS, false, false) DG_X2(SS, true, false) DG_X2(SS, false, true) DG_X2(SS, true, true)
  DG_X2ALL(10) DG_X2ALL(12) DG_X2ALL(14) DG_X2ALL(16)
#undef DG_X2ALL
#undef DG_X2
  return {};
}

}  // namespace dg
