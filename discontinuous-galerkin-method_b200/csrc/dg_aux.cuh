// dg_aux.cuh — layout conversions and diagnostics (fetch, load, halo pack/unpack, energy, watchdog).
#pragma once
#include "dg_common.cuh"

namespace dg {

// -------------------------------------------------------------------------------------------
// Layout conversions and diagnostics.

// internal [plane][e*S+s] (locality order) -> reference element-major double[K][6]
template <class R>
__global__ void k_fetch_field(const R* __restrict__ U, int plane0, long long ES, long long PS, int s,
                              const int* __restrict__ new_of_old, int K, double* __restrict__ out) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)K * NP) return;
  const int eo = (int)(q / NP), i = (int)(q - (long long)eo * NP);
  const int en = __ldg(new_of_old + eo);
  out[q] = (double)U[(long long)en * ES + (plane0 + i) * PS + s];
}

// Halo exchange of a mesh split over several contexts: planes plane0 .. plane0+planes-1 of the
// listed (internal) elements, all S shots, to or from buf[k][plane][s].
template <class R>
__global__ void k_halo_pack(const R* __restrict__ U, long long ES, long long PS, int S, int plane0, int planes,
                            const int* __restrict__ elems, int n, R* __restrict__ buf) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * planes * S) return;
  const int s = (int)(q % S);
  const long long r = q / S;
  const int pl = (int)(r % planes), k = (int)(r / planes);
  buf[q] = U[(long long)__ldg(elems + k) * ES + (long long)(plane0 + pl) * PS + s];
}
template <class R>
__global__ void k_halo_unpack(R* __restrict__ U, long long ES, long long PS, int S, int plane0, int planes,
                              const int* __restrict__ elems, int n, const R* __restrict__ buf) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * planes * S) return;
  const int s = (int)(q % S);
  const long long r = q / S;
  const int pl = (int)(r % planes), k = (int)(r / planes);
  U[(long long)__ldg(elems + k) * ES + (long long)(plane0 + pl) * PS + s] = buf[q];
}

template <class R>
__global__ void k_load_field(R* __restrict__ U, R* __restrict__ C, int plane0, long long ES, long long PS, int s,
                             const int* __restrict__ new_of_old, int K, const double* __restrict__ in) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)K * NP) return;
  const int eo = (int)(q / NP), i = (int)(q - (long long)eo * NP);
  const int en = __ldg(new_of_old + eo);
  const long long at = (long long)en * ES + (plane0 + i) * PS + s;
  U[at] = (R)in[q];
  if (C) C[at] = R(0);
}

template <class R>
__global__ void k_fetch_trace(const R* __restrict__ tr, int comp, int n_rec, int S, int s, long long steps,
                              double* __restrict__ out) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= steps * n_rec) return;
  const long long t = q / n_rec;
  const int r = (int)(q - t * n_rec);
  out[q] = (double)tr[((t * 2 + comp) * n_rec + r) * (long long)S + s];
}

// traces of steps [t0, t0+n) of the first S_out shots (of S_lay stored) -> out_x / out_z [s][t - t0][r]
template <class R>
__global__ void k_fetch_traces(const R* __restrict__ tr, int n_rec, int S_lay, int S_out, long long t0, long long n,
                               double* __restrict__ out_x, double* __restrict__ out_z) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int S = S_out;
  const long long per = n * n_rec * S;
  if (q >= 2 * per) return;
  const int comp = (int)(q / per);
  long long rem = q - comp * per;
  const int s = (int)(rem / (n * n_rec));
  rem -= (long long)s * n * n_rec;
  const long long t = rem / n_rec;
  const int r = (int)(rem - t * n_rec);
  (comp ? out_z : out_x)[q - comp * per] = (double)tr[(((t0 + t) * 2 + comp) * n_rec + r) * (long long)S_lay + s];
}

// 1/2 sum_e J_e sum_ij M_ij [rho v_i.v_j + compliance(sigma_i, sigma_j)], FP64 accumulation.
template <class R>
__global__ void k_energy(const __grid_constant__ Ops<R> ops, const __grid_constant__ MeshDev<R> m, int s,
                         double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double local = 0.0;
  if (e < m.K) {
    const auto gm = m.geo[e];
    const auto mt = m.mat[e];
    const double rx = gm.x, sx = gm.y, rz = gm.z, sz = gm.w;
    const double J = 1.0 / (rx * sz - sx * rz);
    const double rho = 1.0 / (double)mt.x, lam = mt.y, mu = mt.z;
    const long long g = (long long)e * m.ES + s;
    double f[5][NP];
#pragma unroll
    for (int c = 0; c < 5; c++)
#pragma unroll
      for (int i = 0; i < NP; i++) f[c][i] = (double)m.U[g + (c * NP + i) * m.PS];
    const double det = 4.0 * mu * (lam + mu);
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NP; k++) {
        const double Mik = (double)ops.M[i * NP + k];
        double w = rho * (f[0][i] * f[0][k] + f[1][i] * f[1][k]);
        if (mu > 0.0) {
          w += ((lam + 2 * mu) * (f[2][i] * f[2][k] + f[3][i] * f[3][k]) - lam * (f[2][i] * f[3][k] + f[3][i] * f[2][k])) / det +
               f[4][i] * f[4][k] / mu;
        } else if (lam > 0.0) {
          w += (f[2][i] + f[3][i]) * (f[2][k] + f[3][k]) / (4.0 * lam);
        }
        local += 0.5 * J * Mik * w;
      }
  }
  // block reduction
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x + 31) / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(out, v);
  }
}

template <class R>
__global__ void k_nonfinite(const R* __restrict__ U, long long n, int* __restrict__ flag) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int bad = 0;
  for (; q < n; q += stride) bad |= !isfinite((double)U[q]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace dg
