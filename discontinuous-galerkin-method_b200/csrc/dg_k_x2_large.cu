// dg_k_x2_large.cu — instances of the packed kernels for one shot (two elements per thread) and
// for 32, 64 and 128 shots (element-major, plain and Kahan).
#include "dg_kernels.cuh"

namespace dg {

HalfPair<X2Fn> kernels_packed_large(int S, bool kahan) {
  if (S == 1) {
    if (kahan) return {k_velocity_x2e<true>, k_stress_x2e<true>};
    return {k_velocity_x2e<false>, k_stress_x2e<false>};
  }
#define DG_X2(SS, KH) \
  if (S == SS && kahan == KH) return {k_velocity_x2<SS, KH>, k_stress_x2<SS, KH>};
  DG_X2(32, false) DG_X2(32, true) DG_X2(64, false) DG_X2(64, true) DG_X2(128, false) DG_X2(128, true)
#undef DG_X2
  return {};
}

}  // namespace dg
