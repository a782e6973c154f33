// dg_step_wave.cuh — the whole time step (sponge, source, velocity, stress, record) in one launch,
// as a wavefront that keeps the state of the elements in flight in L2.
//
// Elements are numbered in a bandwidth-reducing (reverse Cuthill-McKee) order.  The unit of work
// is one warp's share of the element range (32 threads, two shots each).  A block takes a ticket
// tau (an atomic counter, so tickets follow the order in which blocks start) and each of its warps
// does two pieces of work, with no barrier between them:
//   * the velocity update of its unit in block tau, the receivers of that unit, then publishes
//     flag[unit] = step id;
//   * the stress update of its unit in block tau - L, after waiting until every unit holding one of
//     that unit's elements or their neighbours has published the flag.
// The stress update of a unit overwrites stresses that only those velocity updates read, so the
// in-place update is safe.  L is at least the unit bandwidth in blocks, so a warp only ever waits
// on units of lower or equal tickets, whose warps are running or done and never wait before
// publishing — no cycle, no deadlock, co-residency not required.  Each wait is bounded: past the
// limit (or once any warp gave up) the warp sets the error word and carries on, and the host
// reports the error.  With the lag window in L2, each state value crosses HBM about once per step:
// 30 reads and 30 writes per element and shot instead of the 90 of two separate passes.
#pragma once
#include "dg_common.cuh"
#include "dg_step_x2.cuh"

#ifndef DG_WAVE_MINB
#define DG_WAVE_MINB 2  // resident blocks of DG_WAVE_MAXT threads per SM the register budget is cut for
#endif
#ifndef DG_WAVE_MAXT
#define DG_WAVE_MAXT 256
#endif

namespace dg {

struct Wave {
  int NU;                 // warp units: ceil(K * S/2 / 32)
  int NB;                 // blocks of units: ceil(NU / warps per block)
  int L;                  // lag between a unit's velocity and its stress work, in blocks
  int W;                  // wait-list width (<= 32)
  const int* wait;        // [NU][W] units holding the unit's elements or their neighbours, -1 padded
  unsigned int* vflag;    // [NU] step id (t + 1) once the unit's new velocities are stored
  const int* rec_start;   // [NU + 1] receivers whose element the unit covers:
  const int* rec_list;    //   rec_list[rec_start[u] .. rec_start[u+1])
  unsigned long long* tickets;  // blocks started since step 0: launch t hands out t*G .. t*G + G - 1
  int* error;             // bit 0: a wait reached its limit
  unsigned int spin_limit;
  unsigned long long inv_G;  // floor((2^64 - 1) / G), G = blocks of the launch
  unsigned int* ptk;      // persistent form: [0] next ticket of the step, [1] blocks finished
};

// Receivers of unit u right after its velocity update (Record, OpenMP_Function.c:61-72): each
// thread stores the two shots it has just updated, so it reads back only its own stores.
template <int S>
__device__ __forceinline__ void record_unit(const MeshDev<float>& m, const Wave& w, int u, int r0, int r1,
                                            long long t) {
  constexpr int H = S / 2;
  const int g = u * 32 + (int)(threadIdx.x & 31);
  const int e = g / H, lane = g - e * H;
  float* tx = m.trace + (t * 2) * (long long)m.n_rec * S;
  float* tz = tx + (long long)m.n_rec * S;
  for (int q = r0; q < r1; q++) {
    const int rr = __ldg(w.rec_list + q);
    if (__ldg(m.rec_elem + rr) != e) continue;
    const int node = __ldg(m.rec_node + rr);
    const float2* Ue = reinterpret_cast<const float2*>(m.U) + (long long)e * 30 * H + lane;
    reinterpret_cast<float2*>(tx + (long long)rr * S)[lane] = Ue[node * H];
    reinterpret_cast<float2*>(tz + (long long)rr * S)[lane] = Ue[(6 + node) * H];
  }
}

// Receivers of unit u of the one-shot layout (thread p owns elements 2p and 2p+1 of the
// plane-major U[plane][Kp]): the thread that has just stored an element's velocities records it.
__device__ __forceinline__ void record_unit_e(const MeshDev<float>& m, const Wave& w, int u, int r0, int r1,
                                              long long t) {
  const int p = u * 32 + (int)(threadIdx.x & 31);
  float* tx = m.trace + (t * 2) * (long long)m.n_rec;
  float* tz = tx + m.n_rec;
  for (int q = r0; q < r1; q++) {
    const int rr = __ldg(w.rec_list + q);
    const int e = __ldg(m.rec_elem + rr);
    if ((e >> 1) != p) continue;
    const int node = __ldg(m.rec_node + rr);
    tx[rr] = m.U[(long long)node * m.P + e];
    tz[rr] = m.U[(long long)(6 + node) * m.P + e];
  }
}

// Layouts of the wavefront step: how a block's velocity and stress halves, its receivers and
// the stress half's early loads are done.
template <int S>
struct WaveTwoShots {  // element-major U[e][plane][S], thread g: element g / (S/2), shots 2q, 2q+1
  using Pre = StressConst;
  template <bool KAHAN>
  static __device__ __forceinline__ void velocity(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
    velocity_x2_body<S, KAHAN>(ops, m, lb, t);
  }
  static __device__ __forceinline__ void record(const MeshDev<float>& m, const Wave& w, int u, int r0, int r1,
                                                long long t) {
    record_unit<S>(m, w, u, r0, r1, t);
  }
  // the stress element's constants, requested before the release and the wait, which they
  // overlap (a thread past the last element reads the last element's and discards them)
  static __device__ __forceinline__ Pre prefetch(const MeshDev<float>& m, int lb) {
    const int g = lb * (int)blockDim.x + (int)threadIdx.x;
    return stress_const(m, min(g / (S / 2), m.K - 1));
  }
  template <bool KAHAN>
  static __device__ __forceinline__ void stress(const Ops2& ops, const MeshDev<float>& m, int lb, long long t,
                                                const Pre& sc) {
    constexpr int H = S / 2;
    const int g = lb * (int)blockDim.x + (int)threadIdx.x;
    if (g < m.K * H) stress_x2_core<S, KAHAN, true>(ops, m, g / H, g - (g / H) * H, sc);
  }
};

// The two-shot layout whose halves request the element's own old values (velocities and
// compensations in the velocity half, stresses and compensations in the stress half) into
// shared memory at their start (cp.async, no registers held) and read them from there for the
// update.  Each warp has wave_stage_slots<KAHAN>() float2 per lane of the block's dynamic shared
// memory; the two halves of a ticket reuse them one after the other.
template <bool KAHAN> __host__ __device__ constexpr int wave_stage_slots() { return KAHAN ? 36 : 18; }

template <int S>
struct WaveTwoShotsAsync : WaveTwoShots<S> {
  using Pre = StressConst;
  template <bool KAHAN>
  static __device__ __forceinline__ float2* stage() {
    extern __shared__ float2 wave_stage[];
    return wave_stage + (threadIdx.x >> 5) * (wave_stage_slots<KAHAN>() * 32) + (threadIdx.x & 31);
  }
  template <bool KAHAN>
  static __device__ __forceinline__ void velocity(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
    velocity_x2_body<S, KAHAN, false, true>(ops, m, lb, t, stage<KAHAN>());
  }
  template <bool KAHAN>
  static __device__ __forceinline__ void stress(const Ops2& ops, const MeshDev<float>& m, int lb, long long t,
                                                const Pre& sc) {
    constexpr int H = S / 2;
    const int g = lb * (int)blockDim.x + (int)threadIdx.x;
    if (g < m.K * H) stress_x2_core<S, KAHAN, true, false, true>(ops, m, g / H, g - (g / H) * H, sc, stage<KAHAN>());
  }
};

struct WaveOneShot {  // plane-major U[plane][Kp], thread p: elements 2p and 2p+1
  struct Pre {};
  template <bool KAHAN>
  static __device__ __forceinline__ void velocity(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
    velocity_x2e_body<KAHAN>(ops, m, lb, t);
  }
  static __device__ __forceinline__ void record(const MeshDev<float>& m, const Wave& w, int u, int r0, int r1,
                                                long long t) {
    record_unit_e(m, w, u, r0, r1, t);
  }
  static __device__ __forceinline__ Pre prefetch(const MeshDev<float>&, int) { return {}; }
  template <bool KAHAN>
  static __device__ __forceinline__ void stress(const Ops2& ops, const MeshDev<float>& m, int lb, long long t,
                                                const Pre&) {
    stress_x2e_body<KAHAN, true>(ops, m, lb, t);
  }
};

// Each lane waits on one unit of the wait list (k < 0: none) to publish step id.
__device__ __forceinline__ void wait_units(const Wave& w, int k, unsigned id) {
  if (k >= 0) {
    unsigned spins = 0;
    while (ld_acquire_u32(w.vflag + k) != id) {
      if (++spins > w.spin_limit || (ld_volatile_i32(w.error) & 1)) {
        atomicOr(w.error, 1);
        break;
      }
      __nanosleep(32);
    }
  }
  __syncwarp();
}

// The work of ticket tau in step t: the velocity half of the units of block tau and the stress
// half of the units of block tau - L (each warp one unit of each).
template <class Layout, bool KAHAN>
__device__ __forceinline__ void wave_ticket(const Ops2& ops, const MeshDev<float>& m, const Wave& w, int tau,
                                            long long t) {
  const unsigned id = (unsigned)(t + 1);
  const int wpb = (int)(blockDim.x >> 5), warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const int uv = tau * wpb + warp, j = tau - w.L, ut = j * wpb + warp;
  const bool do_v = tau < w.NB && uv < w.NU;
  const bool do_t = j >= 0 && j < w.NB && ut < w.NU;
  // the stress unit's wait list and the velocity unit's receiver range are fetched before the
  // velocity work, so their latency hides behind it
  const int k = (do_t && lane < w.W) ? __ldg(w.wait + (long long)ut * w.W + lane) : -1;
  int r0 = 0, r1 = 0;
  if (do_v) {
    r0 = __ldg(w.rec_start + uv);
    r1 = __ldg(w.rec_start + uv + 1);
  }
  if (do_v) {
    Layout::template velocity<KAHAN>(ops, m, tau, t);
    __syncwarp();
    if (r0 != r1) Layout::record(m, w, uv, r0, r1, t);
    __syncwarp();
  }
  typename Layout::Pre pre{};
  if (do_t) pre = Layout::prefetch(m, j);
  // the warp barrier above orders every lane's stores before lane 0's release (a release fence
  // and a relaxed store: 0.6103 against 0.6112 ms a step with st.release on the 200k x 64 batch)
  if (do_v && lane == 0) {
    fence_release_gpu();
    st_relaxed_u32(w.vflag + uv, id);
  }
  if (do_t) {
    wait_units(w, k, id);
    Layout::template stress<KAHAN>(ops, m, j, t, pre);
  }
}

template <class Layout, bool KAHAN>
__global__ void __launch_bounds__(DG_WAVE_MAXT, DG_WAVE_MINB) k_step_wave(const __grid_constant__ Ops2 ops,
                                                                 const __grid_constant__ MeshDev<float> m,
                                                                 const __grid_constant__ Wave w,
                                                                 Counters* __restrict__ ctr) {
  __shared__ long long s_t;
  __shared__ int s_tau;
  if (threadIdx.x == 0) {
    // the ticket gives both the step (ticket / G) and the block's place in it, so no block reads
    // the counters and none has to rewind anything at the end of the launch; the quotient comes
    // from the reciprocal, one short of the true one at most
    const unsigned long long tk = atomicAdd(w.tickets, 1ull), G = gridDim.x;
    unsigned long long q = __umul64hi(tk, w.inv_G);
    if (tk - q * G >= G) q++;
    s_t = (long long)q;
    s_tau = (int)(tk - q * G);
  }
  __syncthreads();
  const long long t = s_t;
  const int tau = s_tau;
  if (tau == 0 && threadIdx.x == 0) {
    ctr->v = t + 1;
    ctr->s = t + 1;
  }
  if (t >= m.steps) return;
  wave_ticket<Layout, KAHAN>(ops, m, w, tau, t);
}

// Persistent form: a grid of resident blocks, each taking tickets 0 .. G-1 of the step in turn
// (w.ptk[0]) and asking for its next ticket while it works on the current one.  A block that
// holds an unstarted ticket p is busy with a lower ticket whose stress half waits only on lower
// tickets still, so the waits cannot form a cycle.  The last block to finish (w.ptk[1]) rewinds
// the tickets and advances the step counters; every block reads the counters before it counts
// itself finished, so none sees the new value.
template <class Layout, bool KAHAN>
__global__ void __launch_bounds__(DG_WAVE_MAXT, DG_WAVE_MINB) k_step_wave_p(const __grid_constant__ Ops2 ops,
                                                                   const __grid_constant__ MeshDev<float> m,
                                                                   const __grid_constant__ Wave w,
                                                                   Counters* __restrict__ ctr) {
  __shared__ int s_tau[2];
  const long long t = ctr->v;
  const int G = w.NB + w.L;
  if (t < m.steps) {
    if (threadIdx.x == 0) s_tau[0] = (int)atomicAdd(w.ptk, 1u);
    __syncthreads();
    int cur = s_tau[0];
    for (int it = 0; cur < G; it++) {
      unsigned nxt = 0;
      if (threadIdx.x == 0) nxt = atomicAdd(w.ptk, 1u);  // used only after this ticket's work
      wave_ticket<Layout, KAHAN>(ops, m, w, cur, t);
      if (threadIdx.x == 0) s_tau[(it + 1) & 1] = (int)nxt;
      __syncthreads();
      cur = s_tau[(it + 1) & 1];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(w.ptk + 1, 1u) == gridDim.x - 1) {
      w.ptk[0] = 0u;
      w.ptk[1] = 0u;
      ctr->v = t + 1;
      ctr->s = t + 1;
      __threadfence();
    }
  }
}

}  // namespace dg
