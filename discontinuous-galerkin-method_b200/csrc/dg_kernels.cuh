// dg_kernels.cuh — the step kernels the host code launches, by family, as typed function
// pointers.  Each family's instances live in a translation unit of their own (dg_k_*.cu), which
// take their addresses and so compile them; the host code (dg_gpu.cu) asks for the instance it
// needs here and launches it through the pointer.  A null pointer means "no instance".
#pragma once
#include "dg_common.cuh"
#include "dg_step_multi.cuh"
#include "dg_step_wave.cuh"
#include "dg_step_x2.cuh"

namespace dg {

// k_velocity / k_stress (geometric-factor form, one (element, shot) per thread) and the
// reference-operator kernels k_velocity_ref / k_stress_ref: (ops, one mesh, mesh table, block table, counters)
template <class R> using GenFn = void (*)(Ops<R>, MeshDev<R>, const MeshDev<R>*, const int2*, Counters*);
// the packed one-mesh kernels k_velocity_x2 / k_stress_x2 / k_velocity_x2e / k_stress_x2e
using X2Fn = void (*)(Ops2, MeshDev<float>, Counters*);
// the wavefront step k_step_wave / k_step_wave_p
using WaveFn = void (*)(Ops2, MeshDev<float>, Wave, Counters*);
// the batch kernels k_velocity_mx / k_stress_mx
using MxFn = void (*)(Ops<float>, Ops2, const MeshDev<float>*, const int2*, Counters*);
// the persistent batch k_step_mx_p
using MxpFn = void (*)(Ops<float>, Ops2, const MeshDev<float>*, MxLoop, Counters*, int);

template <class F> struct HalfPair {
  F v = nullptr;  // velocity half
  F s = nullptr;  // stress half (and the receivers)
};

HalfPair<GenFn<double>> kernels_fp64(bool multi);                 // dg_k_generic.cu
HalfPair<GenFn<float>> kernels_fp32(bool kahan, bool multi);      // dg_k_generic.cu
HalfPair<GenFn<double>> kernels_reference(bool multi, bool otf);  // dg_k_generic.cu
// S shots (2..128, powers of two), or S = 1 on the one-shot layout
WaveFn kernel_wave(int S, bool kahan, bool persistent);           // dg_k_wave.cu
// the resident-block form whose halves stage the element's old values in shared memory
// (S = 16 .. 128); dynamic shared memory: wave_stage_slots<kahan>() * 32 float2 per warp
WaveFn kernel_wave_async(int S, bool kahan);                      // dg_k_wave.cu
HalfPair<MxFn> kernels_batch(bool kahan);                         // dg_k_multi.cu
MxpFn kernel_batch_persistent(bool kahan);                        // dg_k_multi.cu

// the packed instances, split by shot count over three translation units
HalfPair<X2Fn> kernels_packed_small(int S, bool kahan, bool pm);  // S = 2..8
HalfPair<X2Fn> kernels_packed_mid(int S, bool kahan, bool pm);    // S = 10..16
HalfPair<X2Fn> kernels_packed_large(int S, bool kahan);           // S = 1, 32, 64, 128

// S stored shots (even; element-major, or plane-major with `pm`), or S = 1: two elements per
// thread on the one-shot plane-major layout
inline HalfPair<X2Fn> kernels_packed(int S, bool kahan, bool pm) {
  if (S >= 2 && S <= 8) return kernels_packed_small(S, kahan, pm);
  if (S >= 10 && S <= 16) return kernels_packed_mid(S, kahan, pm);
  if (pm) return {};
  return kernels_packed_large(S, kahan);
}

}  // namespace dg
