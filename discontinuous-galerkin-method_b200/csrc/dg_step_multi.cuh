// dg_step_multi.cuh — one launch per half-step over a batch of FP32 meshes with their own shot
// counts, time steps and step counts.  Each block belongs to one mesh (block table) and runs the
// kernel body that suits that mesh: two elements per thread for one shot, two shots per thread
// (packed FP32x2, element-major layout) for even shot counts — odd counts above one are padded
// on the host with one silent shot, on element-major or (kind 3) plane-major state — and one
// (element, shot) per thread otherwise.
#pragma once
#include "dg_common.cuh"
#include "dg_step_generic.cuh"
#include "dg_step_x2.cuh"

namespace dg {

#define DG_MX_SHOTS(CALL) \
  CALL(2) CALL(4) CALL(6) CALL(8) CALL(10) CALL(12) CALL(14) CALL(16) CALL(32) CALL(64) CALL(128)
#define DG_MX_PM_SHOTS(CALL) CALL(4) CALL(6) CALL(8) CALL(10) CALL(12) CALL(14) CALL(16)

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_velocity_mx(const __grid_constant__ Ops<float> ops,
                                                        const __grid_constant__ Ops2 ops2,
                                                        const MeshDev<float>* __restrict__ tab,
                                                        const int2* __restrict__ btab,
                                                        Counters* __restrict__ ctr) {
  const int2 b = __ldg(btab + blockIdx.x);
  const MeshDev<float>& m = tab[b.x];
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  if (m.kind == 1) {
    velocity_x2e_body<KAHAN>(ops2, m, b.y, t);
  } else if (m.kind == 2) {
    switch (m.S) {
#define DG_MX_V(SS) \
  case SS:          \
    velocity_x2_body<SS, KAHAN>(ops2, m, b.y, t); \
    break;
      DG_MX_SHOTS(DG_MX_V)
#undef DG_MX_V
      default:
        break;
    }
  } else if (m.kind == 3) {
    switch (m.S) {
#define DG_MX_VP(SS) \
  case SS:           \
    velocity_x2_body<SS, KAHAN, true>(ops2, m, b.y, t); \
    break;
      DG_MX_PM_SHOTS(DG_MX_VP)
#undef DG_MX_VP
      default:
        break;
    }
  } else {
    velocity_body<float, KAHAN>(ops, m, b.y, t);
  }
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_stress_mx(const __grid_constant__ Ops<float> ops,
                                                      const __grid_constant__ Ops2 ops2,
                                                      const MeshDev<float>* __restrict__ tab,
                                                      const int2* __restrict__ btab,
                                                      Counters* __restrict__ ctr) {
  const int2 b = __ldg(btab + blockIdx.x);
  const MeshDev<float>& m = tab[b.x];
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  if (b.y >= m.n_elem_blocks) {
    record(m, b.y - m.n_elem_blocks, t);
    return;
  }
  if (m.kind == 1) {
    stress_x2e_body<KAHAN>(ops2, m, b.y, t);
  } else if (m.kind == 2) {
    switch (m.S) {
#define DG_MX_T(SS) \
  case SS:          \
    stress_x2_body<SS, KAHAN>(ops2, m, b.y, t); \
    break;
      DG_MX_SHOTS(DG_MX_T)
#undef DG_MX_T
      default:
        break;
    }
  } else if (m.kind == 3) {
    switch (m.S) {
#define DG_MX_TP(SS) \
  case SS:           \
    stress_x2_body<SS, KAHAN, false, true>(ops2, m, b.y, t); \
    break;
      DG_MX_PM_SHOTS(DG_MX_TP)
#undef DG_MX_TP
      default:
        break;
    }
  } else {
    stress_body<float, KAHAN>(ops, m, b.y, t);
  }
}

}  // namespace dg
