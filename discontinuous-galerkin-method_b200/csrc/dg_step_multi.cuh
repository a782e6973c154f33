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
#define DG_MX_PM_SHOTS(CALL) CALL(2) CALL(4) CALL(6) CALL(8) CALL(10) CALL(12) CALL(14) CALL(16)

// The velocity half of one block of the batch: block lb of mesh m, in the body of its kind.
template <bool KAHAN>
__device__ __forceinline__ void mx_velocity_block(const Ops<float>& ops, const Ops2& ops2, const MeshDev<float>& m,
                                                  int lb, long long t) {
  if (t >= m.steps) return;
  if (m.kind == 1) {
    velocity_x2e_body<KAHAN>(ops2, m, lb, t);
  } else if (m.kind == 2) {
    switch (m.S) {
#define DG_MX_V(SS) \
  case SS:          \
    velocity_x2_body<SS, KAHAN>(ops2, m, lb, t); \
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
    velocity_x2_body<SS, KAHAN, true>(ops2, m, lb, t); \
    break;
      DG_MX_PM_SHOTS(DG_MX_VP)
#undef DG_MX_VP
      default:
        break;
    }
  } else {
    velocity_body<float, KAHAN>(ops, m, lb, t);
  }
}

// The stress half (or, past the element blocks, the receivers) of one block of the batch.
template <bool KAHAN>
__device__ __forceinline__ void mx_stress_block(const Ops<float>& ops, const Ops2& ops2, const MeshDev<float>& m,
                                                int lb, long long t) {
  if (t >= m.steps) return;
  if (lb >= m.n_elem_blocks) {
    record(m, lb - m.n_elem_blocks, t);
    return;
  }
  if (m.kind == 1) {
    stress_x2e_body<KAHAN>(ops2, m, lb, t);
  } else if (m.kind == 2) {
    switch (m.S) {
#define DG_MX_T(SS) \
  case SS:          \
    stress_x2_body<SS, KAHAN>(ops2, m, lb, t); \
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
    stress_x2_body<SS, KAHAN, false, true>(ops2, m, lb, t); \
    break;
      DG_MX_PM_SHOTS(DG_MX_TP)
#undef DG_MX_TP
      default:
        break;
    }
  } else {
    stress_body<float, KAHAN>(ops, m, lb, t);
  }
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_velocity_mx(const __grid_constant__ Ops<float> ops,
                                                        const __grid_constant__ Ops2 ops2,
                                                        const MeshDev<float>* __restrict__ tab,
                                                        const int2* __restrict__ btab,
                                                        Counters* __restrict__ ctr) {
  pdl_enter();
  const int2 b = __ldg(btab + blockIdx.x);
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  mx_velocity_block<KAHAN>(ops, ops2, tab[b.x], b.y, t);
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_stress_mx(const __grid_constant__ Ops<float> ops,
                                                      const __grid_constant__ Ops2 ops2,
                                                      const MeshDev<float>* __restrict__ tab,
                                                      const int2* __restrict__ btab,
                                                      Counters* __restrict__ ctr) {
  pdl_enter();
  const int2 b = __ldg(btab + blockIdx.x);
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  mx_stress_block<KAHAN>(ops, ops2, tab[b.x], b.y, t);
}

// -------------------------------------------------------------------------------------------
// The batch's time loop in one persistent launch: a cooperative grid of resident blocks runs
// `nsteps` steps; in each half every block takes the work blocks of the block table in turn
// (the same bodies as the two launches above), and a grid barrier separates the halves.  The
// barrier follows the pattern of a cooperative-groups grid sync (block barrier; thread 0:
// fence, arrive, wait for the generation to change, fence; block barrier), so the loads after
// it see every store before it.  Its wait is bounded: past the limit (or once another block
// gave up) the block sets bit 1 of the error word and the kernel ends.
struct MxLoop {
  const int2* btab_v;  // work blocks of the velocity half: (mesh, block)
  const int2* btab_t;  // of the stress half, recorder blocks included
  int nv, nt;
  unsigned* bar;       // [0] arrivals, [1] generation (arrivals zero at launch)
  int* error;
  unsigned spin_limit;
  unsigned extra;      // arrivals expected beyond the grid: 0 (1 only in a test that makes the wait run out)
};

__device__ __forceinline__ bool grid_barrier(const MxLoop& L) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned gen = ld_acquire_u32(L.bar + 1);
    __threadfence();
    if (atomicAdd(L.bar, 1u) == gridDim.x - 1 + L.extra) {
      L.bar[0] = 0u;
      st_release_u32(L.bar + 1, gen + 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire_u32(L.bar + 1) == gen) {
        if (++spins > L.spin_limit || (ld_volatile_i32(L.error) & 2)) {
          atomicOr(L.error, 2);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_step_mx_p(const __grid_constant__ Ops<float> ops,
                                                      const __grid_constant__ Ops2 ops2,
                                                      const MeshDev<float>* __restrict__ tab,
                                                      const __grid_constant__ MxLoop L,
                                                      Counters* __restrict__ ctr, int nsteps) {
  const long long t0 = ctr->v;
  for (int s = 0; s < nsteps; s++) {
    const long long t = t0 + s;
    for (int w = blockIdx.x; w < L.nv; w += gridDim.x) {
      const int2 b = __ldg(L.btab_v + w);
      mx_velocity_block<KAHAN>(ops, ops2, tab[b.x], b.y, t);
    }
    if (!grid_barrier(L)) return;
    for (int w = blockIdx.x; w < L.nt; w += gridDim.x) {
      const int2 b = __ldg(L.btab_t + w);
      mx_stress_block<KAHAN>(ops, ops2, tab[b.x], b.y, t);
    }
    if (!grid_barrier(L)) return;
  }
  // every block read t0 before the first barrier, so the counters can move now
  if (blockIdx.x == 0 && threadIdx.x == 0 && nsteps > 0) {
    ctr->v = t0 + nsteps;
    ctr->s = t0 + nsteps - 1;
  }
}

}  // namespace dg
