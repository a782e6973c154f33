// dg_k_multi.cu — instances of the batch kernels: two launches a step (k_velocity_mx /
// k_stress_mx) and the persistent cooperative form (k_step_mx_p), plain and Kahan.  Each of
// these kernels dispatches to every packed body, so the file is compiled once per instance
// (DG_MX_PART 1..6, one instance each, in parallel) and once for the getters (DG_MX_PART 0).
#include "dg_kernels.cuh"

#ifndef DG_MX_PART
#define DG_MX_PART 0
#endif

namespace dg {

MxFn mx_velocity_plain();     // part 1
MxFn mx_velocity_kahan();     // part 2
MxFn mx_stress_plain();       // part 3
MxFn mx_stress_kahan();       // part 4
MxpFn mx_persistent_plain();  // part 5
MxpFn mx_persistent_kahan();  // part 6

#if DG_MX_PART == 0
HalfPair<MxFn> kernels_batch(bool kahan) {
  if (kahan) return {mx_velocity_kahan(), mx_stress_kahan()};
  return {mx_velocity_plain(), mx_stress_plain()};
}
MxpFn kernel_batch_persistent(bool kahan) { return kahan ? mx_persistent_kahan() : mx_persistent_plain(); }
#elif DG_MX_PART == 1
MxFn mx_velocity_plain() { return k_velocity_mx<false>; }
#elif DG_MX_PART == 2
MxFn mx_velocity_kahan() { return k_velocity_mx<true>; }
#elif DG_MX_PART == 3
MxFn mx_stress_plain() { return k_stress_mx<false>; }
#elif DG_MX_PART == 4
MxFn mx_stress_kahan() { return k_stress_mx<true>; }
#elif DG_MX_PART == 5
MxpFn mx_persistent_plain() { return k_step_mx_p<false>; }
#elif DG_MX_PART == 6
MxpFn mx_persistent_kahan() { return k_step_mx_p<true>; }
#endif

}  // namespace dg
