// dg_k_generic.cu — instances of the geometric-factor kernels (FP64, FP32, FP32-Kahan; one mesh
// or a batch) and of the reference-operator kernels.
#include "dg_kernels.cuh"
#include "dg_step_generic.cuh"
#include "dg_step_ref.cuh"

namespace dg {

HalfPair<GenFn<double>> kernels_fp64(bool multi) {
  if (multi) return {k_velocity<double, false, true>, k_stress<double, false, true>};
  return {k_velocity<double, false, false>, k_stress<double, false, false>};
}

HalfPair<GenFn<float>> kernels_fp32(bool kahan, bool multi) {
  if (kahan) {
    if (multi) return {k_velocity<float, true, true>, k_stress<float, true, true>};
    return {k_velocity<float, true, false>, k_stress<float, true, false>};
  }
  if (multi) return {k_velocity<float, false, true>, k_stress<float, false, true>};
  return {k_velocity<float, false, false>, k_stress<float, false, false>};
}

HalfPair<GenFn<double>> kernels_reference(bool multi, bool otf) {
  if (multi) return {k_velocity_ref<true, false>, k_stress_ref<true, false>};
  if (otf) return {k_velocity_ref<false, true>, k_stress_ref<false, true>};
  return {k_velocity_ref<false, false>, k_stress_ref<false, false>};
}

}  // namespace dg
