// dg_step_x2.cuh — two-shot FP32 step kernels on packed FP32x2 arithmetic.
#pragma once
#include "dg_common.cuh"

namespace dg {

// -------------------------------------------------------------------------------------------
// Two-shot FP32 kernels for even shot counts, on Blackwell's packed FP32x2 arithmetic
// (__ffma2_rn / __fmul2_rn / __fadd2_rn: one instruction advances two shots).  Layout:
// element-major with shots innermost, U[e][plane][S], so thread q of an element owns shots 2q and
// 2q+1 as one float2 and all 30 planes of its element sit at compile-time offsets (multiples of
// S/2 float2) from one base address; a neighbour's planes likewise from nb * 30 * S/2.  The
// operators are the compile-time P2 tables (p2_dr, p2_ds, p2_lift), so no operator value is
// loaded at run time.
struct Ops2 {
  float2 Dr[NP * NP];
  float2 Ds[NP * NP];
  float2 L[NF * NP * NF];
};

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, exactly rounded (b * -1 is exact)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// h + c x for an operator entry c known at compile time: nothing for 0, an add or a subtract for
// +-1 (the same rounding as the FMA), a packed FMA otherwise
__device__ __forceinline__ float2 axpy_c(float c, float2 x, float2 h) {
  if (c == 0.f) return h;
  if (c == 1.f) return add2(h, x);
  if (c == -1.f) return sub2(h, x);
  return fma2(f2(c), x, h);
}

// Kahan-compensated u += d with compensation c (both lanes)
__device__ __forceinline__ void kahan2(float2& u, float2& c, float2 d) {
  const float2 y = sub2(d, c);
  const float2 t = add2(u, y);
  c = sub2(sub2(t, u), y);
  u = t;
}

// Bodies take the mesh, the block's index within that mesh and the step; the __global__
// wrappers below (one mesh) and the multi-mesh dispatchers (dg_step_multi.cuh) call them.
// PM: plane-major layout U[plane][e*S + s] (plane stride Kp*S/2 float2) instead of the
// element-major U[e][plane][S]; the arithmetic is the same.
// ASYNC (the wavefront step): the element's own velocities (and compensations) are requested at
// the start into this thread's slots of `stage` (stage[plane * 32], cp.async: no registers held)
// and read from there for the update, so their round trip overlaps the stress loads'.
template <int S, bool KAHAN, bool PM = false, bool ASYNC = false>
__device__ __forceinline__ void velocity_x2_body(const Ops2& ops, const MeshDev<float>& m, int lb, long long t,
                                                 float2* stage = nullptr) {
  constexpr int H = S / 2;    // float2 lanes per element
  constexpr int ES = 30 * H;  // element stride in float2 (element-major)
  const long long EO = PM ? H : ES;                   // element offset
  const long long PS = PM ? (long long)m.Kp * H : H;  // plane stride
  const int g = lb * blockDim.x + threadIdx.x;
  if (g >= m.K * H) return;
  const int e = g / H, q = g - e * H;
  float2* __restrict__ Ue = reinterpret_cast<float2*>(m.U) + (long long)e * EO + q;
  if constexpr (ASYNC) {
#pragma unroll
    for (int i = 0; i < 12; i++) cp_async8(stage + i * 32, Ue + i * PS);
    if (KAHAN) {
      const float2* Ce0 = reinterpret_cast<const float2*>(m.C) + (long long)e * EO + q;
#pragma unroll
      for (int i = 0; i < 12; i++) cp_async8(stage + (12 + i) * 32, Ce0 + i * PS);
    }
    cp_async_commit();
  }

  float2 txx[NP], tzz[NP], txz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    txx[i] = Ue[(12 + i) * PS];
    tzz[i] = Ue[(18 + i) * PS];
    txz[i] = Ue[(24 + i) * PS];
  }
  const int4 fc = __ldg(m.face + e);
  const float4 gm = __ldg(m.geo + e);
  const float irho = __ldg(&m.mat[e].x);
  const bool own_sponge = fc.w & 1;
  if (own_sponge) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const float2 a = f2(__ldg(m.sponge + (long long)i * m.Kp + e));
      txx[i] = mul2(txx[i], a); tzz[i] = mul2(tzz[i], a); txz[i] = mul2(txz[i], a);
    }
  }
  float2 hx[NP], hz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { hx[i] = f2(0.f); hz[i] = f2(0.f); }

  // surface terms: sum_j S_j (nx_j dTxx + nz_j dTxz), sum_j S_j (nz_j dTzz + nx_j dTxz)
  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    float nxs, nzs;
    if (j == 0) { nxs = -0.5f * gm.y; nzs = -0.5f * gm.w; }
    else if (j == 1) { nxs = 0.5f * (gm.x + gm.y); nzs = 0.5f * (gm.z + gm.w); }
    else { nxs = -0.5f * gm.x; nzs = -0.5f * gm.z; }
    const float2 nx = f2(nxs), nz = f2(nzs);
    float2 pxx[NF], pzz[NF], pxz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { pxx[k] = f2(0.f); pzz[k] = f2(0.f); pxz[k] = f2(0.f); }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const float2* __restrict__ Un = reinterpret_cast<const float2*>(m.U) + (long long)nb * EO + q;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        pxx[k] = Un[(12 + node) * PS];
        pzz[k] = Un[(18 + node) * PS];
        pxz[k] = Un[(24 + node) * PS];
      }
      if (code & 8) {
#pragma unroll
        for (int k = 0; k < NF; k++) {
          const int node = face_node(nf, flip ? 2 - k : k);
          const float2 a = f2(__ldg(m.sponge + (long long)node * m.Kp + nb));
          pxx[k] = mul2(pxx[k], a); pzz[k] = mul2(pzz[k], a); pxz[k] = mul2(pxz[k], a);
        }
      }
    }
    float2 fx[NF], fz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const float2 dxx = sub2(pxx[k], txx[own]);
      const float2 dzz = sub2(pzz[k], tzz[own]);
      const float2 dxz = sub2(pxz[k], txz[own]);
      fx[k] = fma2(nx, dxx, mul2(nz, dxz));
      fz[k] = fma2(nz, dzz, mul2(nx, dxz));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        hx[i] = axpy_c(p2_lift((j * NP + i) * NF + k), fx[k], hx[i]);
        hz[i] = axpy_c(p2_lift((j * NP + i) * NF + k), fz[k], hz[i]);
      }
  }

  // volume terms: Dr (rx Txx + rz Txz) + Ds (sx Txx + sz Txz) and the same for (Txz, Tzz); each
  // nonzero operator entry is read once and serves both components
  const float2 rx = f2(gm.x), sx = f2(gm.y), rz = f2(gm.z), sz = f2(gm.w);
  {
    float2 a[NP], b[NP], c[NP], d[NP];
#pragma unroll
    for (int n = 0; n < NP; n++) {
      a[n] = fma2(rx, txx[n], mul2(rz, txz[n]));
      b[n] = fma2(sx, txx[n], mul2(sz, txz[n]));
      c[n] = fma2(rx, txz[n], mul2(rz, tzz[n]));
      d[n] = fma2(sx, txz[n], mul2(sz, tzz[n]));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int n = 0; n < NP; n++) {
        hx[i] = axpy_c(p2_dr(i * NP + n), a[n], hx[i]);
        hz[i] = axpy_c(p2_dr(i * NP + n), c[n], hz[i]);
        hx[i] = axpy_c(p2_ds(i * NP + n), b[n], hx[i]);
        hz[i] = axpy_c(p2_ds(i * NP + n), d[n], hz[i]);
      }
  }

  // V = a V (+ source on Vz) + dt/rho * rhs
  float2 vx[NP], vz[NP], cx[NP], cz[NP];
  float2* __restrict__ Ce = nullptr;
  if (KAHAN) Ce = reinterpret_cast<float2*>(m.C) + (long long)e * EO + q;
  if constexpr (ASYNC) {
    cp_async_wait_all();
#pragma unroll
    for (int i = 0; i < NP; i++) { vx[i] = stage[(0 + i) * 32]; vz[i] = stage[(6 + i) * 32]; }
    if (KAHAN) {
#pragma unroll
      for (int i = 0; i < NP; i++) { cx[i] = stage[(12 + i) * 32]; cz[i] = stage[(18 + i) * 32]; }
    }
  } else {
#pragma unroll
    for (int i = 0; i < NP; i++) { vx[i] = Ue[(0 + i) * PS]; vz[i] = Ue[(6 + i) * PS]; }
    if (KAHAN) {
#pragma unroll
      for (int i = 0; i < NP; i++) { cx[i] = Ce[(0 + i) * PS]; cz[i] = Ce[(6 + i) * PS]; }
    }
  }
  if (own_sponge) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const float2 a = f2(__ldg(m.sponge + (long long)i * m.Kp + e));
      vx[i] = mul2(vx[i], a); vz[i] = mul2(vz[i], a);
      if (KAHAN) { cx[i] = mul2(cx[i], a); cz[i] = mul2(cz[i], a); }
    }
  }
  const int2 se = __ldg(reinterpret_cast<const int2*>(m.src_elem) + q);
  float2 src[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) src[i] = f2(0.f);
  if (se.x == e || se.y == e) {
    const float w = (float)__ldg(m.wavelet + t);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      src[i].x = se.x == e ? __ldg(m.src_fun + (2 * q) * NP + i) * w : 0.f;
      src[i].y = se.y == e ? __ldg(m.src_fun + (2 * q + 1) * NP + i) * w : 0.f;
    }
  }
  const float2 step = f2(m.dt * irho);
#pragma unroll
  for (int i = 0; i < NP; i++) {
    if (KAHAN) {
      kahan2(vx[i], cx[i], mul2(step, hx[i]));
      kahan2(vz[i], cz[i], fma2(step, hz[i], src[i]));
    } else {
      vx[i] = fma2(step, hx[i], vx[i]);
      vz[i] = fma2(step, hz[i], add2(vz[i], src[i]));
    }
    Ue[(0 + i) * PS] = vx[i];
    Ue[(6 + i) * PS] = vz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { Ce[(0 + i) * PS] = cx[i]; Ce[(6 + i) * PS] = cz[i]; }
  }
}

template <int S, bool KAHAN, bool PM = false>
__global__ void __launch_bounds__(256, 2) k_velocity_x2(const __grid_constant__ Ops2 ops,
                                                        const __grid_constant__ MeshDev<float> m,
                                                        Counters* __restrict__ ctr) {
  pdl_enter();
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  velocity_x2_body<S, KAHAN, PM>(ops, m, blockIdx.x + m.block0, t);
}

// Load of a velocity value: plain, or through L2 (FRESH) when other blocks of the same launch
// wrote it (the wavefront step), so no stale L1 line can be returned.
template <bool FRESH>
__device__ __forceinline__ float2 ld_v(const float2* p) {
  if (FRESH) return __ldcg(p);
  return *p;
}

// The per-element constants of the stress update: face codes, geometric factors, materials.
struct StressConst {
  int4 fc;
  float4 gm, mt;
};
__device__ __forceinline__ StressConst stress_const(const MeshDev<float>& m, int e) {
  return {__ldg(m.face + e), __ldg(m.geo + e), __ldg(m.mat + e)};
}

// Stress update of lane q (shots 2q, 2q+1) of element e with its constants already loaded.
// ASYNC: the element's own stresses (and compensations) are requested at the start into this
// thread's slots of `stage` and read from there for the update (see velocity_x2_body).
template <int S, bool KAHAN, bool FRESH, bool PM = false, bool ASYNC = false>
__device__ __forceinline__ void stress_x2_core(const Ops2& ops, const MeshDev<float>& m, int e, int q,
                                               const StressConst& k, float2* stage = nullptr) {
  constexpr int H = S / 2;
  constexpr int ES = 30 * H;
  const long long EO = PM ? H : ES;                   // element offset
  const long long PS = PM ? (long long)m.Kp * H : H;  // plane stride
  float2* __restrict__ Ue = reinterpret_cast<float2*>(m.U) + (long long)e * EO + q;
  if constexpr (ASYNC) {
#pragma unroll
    for (int i = 0; i < 18; i++) cp_async8(stage + i * 32, Ue + (12 + i) * PS);
    if (KAHAN) {
      const float2* Ce0 = reinterpret_cast<const float2*>(m.C) + (long long)e * EO + q;
#pragma unroll
      for (int i = 0; i < 18; i++) cp_async8(stage + (18 + i) * 32, Ce0 + (12 + i) * PS);
    }
    cp_async_commit();
  }

  float2 vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = ld_v<FRESH>(Ue + (0 + i) * PS); vz[i] = ld_v<FRESH>(Ue + (6 + i) * PS); }
  const int4 fc = k.fc;
  const float4 gm = k.gm;
  const float4 mt = k.mt;
  const float2 rx = f2(gm.x), sx = f2(gm.y), rz = f2(gm.z), sz = f2(gm.w);

  // volume: X = dxVx, Z = dzVz, W = dxVz + dzVx
  float2 X[NP], Z[NP], W[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    float2 drx = f2(0.f), dsx = f2(0.f), drz = f2(0.f), dsz = f2(0.f);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      drx = axpy_c(p2_dr(i * NP + n), vx[n], drx);
      drz = axpy_c(p2_dr(i * NP + n), vz[n], drz);
      dsx = axpy_c(p2_ds(i * NP + n), vx[n], dsx);
      dsz = axpy_c(p2_ds(i * NP + n), vz[n], dsz);
    }
    X[i] = fma2(rx, drx, mul2(sx, dsx));
    Z[i] = fma2(rz, drz, mul2(sz, dsz));
    W[i] = fma2(rx, drz, fma2(sx, dsz, fma2(rz, drx, mul2(sz, dsx))));
  }

  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    float nxs, nzs;
    if (j == 0) { nxs = -0.5f * gm.y; nzs = -0.5f * gm.w; }
    else if (j == 1) { nxs = 0.5f * (gm.x + gm.y); nzs = 0.5f * (gm.z + gm.w); }
    else { nxs = -0.5f * gm.x; nzs = -0.5f * gm.z; }
    const float2 nx = f2(nxs), nz = f2(nzs);
    float2 px[NF], pz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { px[k] = f2(0.f); pz[k] = f2(0.f); }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const float2* __restrict__ Un = reinterpret_cast<const float2*>(m.U) + (long long)nb * EO + q;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        px[k] = ld_v<FRESH>(Un + (0 + node) * PS);
        pz[k] = ld_v<FRESH>(Un + (6 + node) * PS);
      }
    }
    float2 fa[NF], fb[NF], fw[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const float2 dvx = sub2(px[k], vx[own]);
      const float2 dvz = sub2(pz[k], vz[own]);
      fa[k] = mul2(nx, dvx);
      fb[k] = mul2(nz, dvz);
      fw[k] = fma2(nz, dvx, mul2(nx, dvz));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const float l = p2_lift((j * NP + i) * NF + k);
        X[i] = axpy_c(l, fa[k], X[i]);
        Z[i] = axpy_c(l, fb[k], Z[i]);
        W[i] = axpy_c(l, fw[k], W[i]);
      }
  }

  float2 txx[NP], tzz[NP], txz[NP], cxx[NP], czz[NP], cxz[NP];
  float2* __restrict__ Ce = nullptr;
  if (KAHAN) Ce = reinterpret_cast<float2*>(m.C) + (long long)e * EO + q;
  if constexpr (ASYNC) {
    cp_async_wait_all();
#pragma unroll
    for (int i = 0; i < NP; i++) {
      txx[i] = stage[(0 + i) * 32];
      tzz[i] = stage[(6 + i) * 32];
      txz[i] = stage[(12 + i) * 32];
    }
    if (KAHAN) {
#pragma unroll
      for (int i = 0; i < NP; i++) {
        cxx[i] = stage[(18 + i) * 32]; czz[i] = stage[(24 + i) * 32]; cxz[i] = stage[(30 + i) * 32];
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      txx[i] = Ue[(12 + i) * PS];
      tzz[i] = Ue[(18 + i) * PS];
      txz[i] = Ue[(24 + i) * PS];
    }
    if (KAHAN) {
#pragma unroll
      for (int i = 0; i < NP; i++) { cxx[i] = Ce[(12 + i) * PS]; czz[i] = Ce[(18 + i) * PS]; cxz[i] = Ce[(24 + i) * PS]; }
    }
  }
  if (fc.w & 1) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const float2 a = f2(__ldg(m.sponge + (long long)i * m.Kp + e));
      txx[i] = mul2(txx[i], a); tzz[i] = mul2(tzz[i], a); txz[i] = mul2(txz[i], a);
      if (KAHAN) { cxx[i] = mul2(cxx[i], a); czz[i] = mul2(czz[i], a); cxz[i] = mul2(cxz[i], a); }
    }
  }
  const float2 dl2m = f2(m.dt * mt.w), dlam = f2(m.dt * mt.y), dmu = f2(m.dt * mt.z);
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const float2 dxx = fma2(dl2m, X[i], mul2(dlam, Z[i]));
    const float2 dzz = fma2(dlam, X[i], mul2(dl2m, Z[i]));
    const float2 dxz = mul2(dmu, W[i]);
    if (KAHAN) {
      kahan2(txx[i], cxx[i], dxx);
      kahan2(tzz[i], czz[i], dzz);
      kahan2(txz[i], cxz[i], dxz);
    } else {
      txx[i] = add2(txx[i], dxx);
      tzz[i] = add2(tzz[i], dzz);
      txz[i] = add2(txz[i], dxz);
    }
    Ue[(12 + i) * PS] = txx[i];
    Ue[(18 + i) * PS] = tzz[i];
    Ue[(24 + i) * PS] = txz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      Ce[(12 + i) * PS] = cxx[i]; Ce[(18 + i) * PS] = czz[i]; Ce[(24 + i) * PS] = cxz[i];
    }
  }
}

template <int S, bool KAHAN, bool FRESH = false, bool PM = false>
__device__ __forceinline__ void stress_x2_body(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
  constexpr int H = S / 2;
  const int g = lb * blockDim.x + threadIdx.x;
  if (g >= m.K * H) return;
  const int e = g / H, q = g - e * H;
  stress_x2_core<S, KAHAN, FRESH, PM>(ops, m, e, q, stress_const(m, e));
}

template <int S, bool KAHAN, bool PM = false>
__global__ void __launch_bounds__(256, 2) k_stress_x2(const __grid_constant__ Ops2 ops,
                                                      const __grid_constant__ MeshDev<float> m,
                                                      Counters* __restrict__ ctr) {
  pdl_enter();
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  const int lb = blockIdx.x + m.block0;
  if (lb >= m.n_elem_blocks) { record(m, lb - m.n_elem_blocks, t); return; }
  stress_x2_body<S, KAHAN, false, PM>(ops, m, lb, t);
}

// -------------------------------------------------------------------------------------------
// Two-element FP32 kernels for one shot: the plane-major layout U[plane][Kp] read as float2, so
// thread p advances elements 2p and 2p+1 with packed arithmetic.  Geometry, materials and face
// codes differ per lane; the neighbour gathers are per lane.  Padding elements (K <= e < Kp)
// carry zero geometry and material, so they compute zeros and stay zero.

__device__ __forceinline__ int pick(const int4& f, int j) { return j == 0 ? f.x : (j == 1 ? f.y : f.z); }

// Decode one lane's face code into a load address that is always valid (element 0 across an
// outer face), the neighbour's three face nodes in our order, a 0/1 mask and the sponge flag,
// so all gathers of a face can be issued without branches.
struct FaceLane {
  int nb;
  int node[NF];
  float mask;
  bool sponge;
};
__device__ __forceinline__ FaceLane face_lane(int code) {
  FaceLane f;
  const bool v = code >= 0;
  f.nb = v ? (code >> 4) : 0;
  const int nf = v ? ((code >> 1) & 3) : 0, fl = v ? (code & 1) : 0;
#pragma unroll
  for (int k = 0; k < NF; k++) f.node[k] = face_node(nf, fl ? 2 - k : k);
  f.mask = v ? 1.f : 0.f;
  f.sponge = v && (code & 8);
  return f;
}
// FRESH: values other blocks of the same launch wrote (the wavefront step), read through L2
template <bool FRESH = false>
__device__ __forceinline__ float2 gather_pair(const MeshDev<float>& m, const FaceLane& a, const FaceLane& b, int pl,
                                              int k) {
  const float* pa = m.U + (long long)(pl + a.node[k]) * m.P + a.nb;
  const float* pb = m.U + (long long)(pl + b.node[k]) * m.P + b.nb;
  if (FRESH) return make_float2(__ldcg(pa) * a.mask, __ldcg(pb) * b.mask);
  return make_float2(*pa * a.mask, *pb * b.mask);
}

template <bool KAHAN>
__device__ __forceinline__ void velocity_x2e_body(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
  const int p = lb * blockDim.x + threadIdx.x;
  const int H = m.Kp / 2;  // plane stride in float2
  if (p >= H) return;
  const int e0 = 2 * p, e1 = 2 * p + 1;
  float2* __restrict__ Up = reinterpret_cast<float2*>(m.U) + p;

  const int4 f0 = __ldg(m.face + e0), f1 = __ldg(m.face + e1);
  const float4 g0 = __ldg(m.geo + e0), g1 = __ldg(m.geo + e1);
  const float2 rx = make_float2(g0.x, g1.x), sx = make_float2(g0.y, g1.y);
  const float2 rz = make_float2(g0.z, g1.z), sz = make_float2(g0.w, g1.w);
  const bool any_sponge = (f0.w | f1.w) & 1;
  float2 sp[NP];
#pragma unroll
  for (int i = 0; i < NP; i++)
    sp[i] = any_sponge ? __ldg(reinterpret_cast<const float2*>(m.sponge + (long long)i * m.Kp) + p) : f2(1.f);

  float2 txx[NP], tzz[NP], txz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    txx[i] = mul2(Up[(12 + i) * H], sp[i]);
    tzz[i] = mul2(Up[(18 + i) * H], sp[i]);
    txz[i] = mul2(Up[(24 + i) * H], sp[i]);
  }
  float2 hx[NP], hz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { hx[i] = f2(0.f); hz[i] = f2(0.f); }
#pragma unroll
  for (int j = 0; j < NF; j++) {
    float2 nx, nz;
    if (j == 0) { nx = mul2(f2(-0.5f), sx); nz = mul2(f2(-0.5f), sz); }
    else if (j == 1) { nx = mul2(f2(0.5f), add2(rx, sx)); nz = mul2(f2(0.5f), add2(rz, sz)); }
    else { nx = mul2(f2(-0.5f), rx); nz = mul2(f2(-0.5f), rz); }
    const FaceLane a = face_lane(pick(f0, j)), b = face_lane(pick(f1, j));
    float2 pxx[NF], pzz[NF], pxz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      pxx[k] = gather_pair(m, a, b, 12, k);
      pzz[k] = gather_pair(m, a, b, 18, k);
      pxz[k] = gather_pair(m, a, b, 24, k);
    }
    if (a.sponge || b.sponge) {
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const float2 w = make_float2(a.sponge ? __ldg(m.sponge + (long long)a.node[k] * m.Kp + a.nb) : 1.f,
                                     b.sponge ? __ldg(m.sponge + (long long)b.node[k] * m.Kp + b.nb) : 1.f);
        pxx[k] = mul2(pxx[k], w); pzz[k] = mul2(pzz[k], w); pxz[k] = mul2(pxz[k], w);
      }
    }
    float2 fx[NF], fz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const float2 dxx = sub2(pxx[k], txx[own]);
      const float2 dzz = sub2(pzz[k], tzz[own]);
      const float2 dxz = sub2(pxz[k], txz[own]);
      fx[k] = fma2(nx, dxx, mul2(nz, dxz));
      fz[k] = fma2(nz, dzz, mul2(nx, dxz));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        hx[i] = axpy_c(p2_lift((j * NP + i) * NF + k), fx[k], hx[i]);
        hz[i] = axpy_c(p2_lift((j * NP + i) * NF + k), fz[k], hz[i]);
      }
  }
  {
    float2 a[NP], b[NP], c[NP], d[NP];
#pragma unroll
    for (int n = 0; n < NP; n++) {
      a[n] = fma2(rx, txx[n], mul2(rz, txz[n]));
      b[n] = fma2(sx, txx[n], mul2(sz, txz[n]));
      c[n] = fma2(rx, txz[n], mul2(rz, tzz[n]));
      d[n] = fma2(sx, txz[n], mul2(sz, tzz[n]));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int n = 0; n < NP; n++) {
        hx[i] = axpy_c(p2_dr(i * NP + n), a[n], hx[i]);
        hz[i] = axpy_c(p2_dr(i * NP + n), c[n], hz[i]);
        hx[i] = axpy_c(p2_ds(i * NP + n), b[n], hx[i]);
        hz[i] = axpy_c(p2_ds(i * NP + n), d[n], hz[i]);
      }
  }
  float2 vx[NP], vz[NP], cx[NP], cz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = mul2(Up[(0 + i) * H], sp[i]); vz[i] = mul2(Up[(6 + i) * H], sp[i]); }
  float2* __restrict__ Cp = nullptr;
  if (KAHAN) {
    Cp = reinterpret_cast<float2*>(m.C) + p;
#pragma unroll
    for (int i = 0; i < NP; i++) { cx[i] = mul2(Cp[(0 + i) * H], sp[i]); cz[i] = mul2(Cp[(6 + i) * H], sp[i]); }
  }
  const int se = __ldg(m.src_elem);
  float2 src[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) src[i] = f2(0.f);
  if (se == e0 || se == e1) {
    const float w = (float)__ldg(m.wavelet + t);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const float v = __ldg(m.src_fun + i) * w;
      src[i] = se == e0 ? make_float2(v, 0.f) : make_float2(0.f, v);
    }
  }
  const float2 step = make_float2(m.dt * __ldg(&m.mat[e0].x), m.dt * __ldg(&m.mat[e1].x));
#pragma unroll
  for (int i = 0; i < NP; i++) {
    if (KAHAN) {
      kahan2(vx[i], cx[i], mul2(step, hx[i]));
      kahan2(vz[i], cz[i], fma2(step, hz[i], src[i]));
    } else {
      vx[i] = fma2(step, hx[i], vx[i]);
      vz[i] = fma2(step, hz[i], add2(vz[i], src[i]));
    }
    Up[(0 + i) * H] = vx[i];
    Up[(6 + i) * H] = vz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { Cp[(0 + i) * H] = cx[i]; Cp[(6 + i) * H] = cz[i]; }
  }
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_velocity_x2e(const __grid_constant__ Ops2 ops,
                                                         const __grid_constant__ MeshDev<float> m,
                                                         Counters* __restrict__ ctr) {
  pdl_enter();
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  velocity_x2e_body<KAHAN>(ops, m, blockIdx.x + m.block0, t);
}

template <bool KAHAN, bool FRESH = false>
__device__ __forceinline__ void stress_x2e_body(const Ops2& ops, const MeshDev<float>& m, int lb, long long t) {
  const int p = lb * blockDim.x + threadIdx.x;
  const int H = m.Kp / 2;
  if (p >= H) return;
  const int e0 = 2 * p, e1 = 2 * p + 1;
  float2* __restrict__ Up = reinterpret_cast<float2*>(m.U) + p;

  float2 vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = ld_v<FRESH>(Up + (0 + i) * H); vz[i] = ld_v<FRESH>(Up + (6 + i) * H); }
  const int4 f0 = __ldg(m.face + e0), f1 = __ldg(m.face + e1);
  const float4 g0 = __ldg(m.geo + e0), g1 = __ldg(m.geo + e1);
  const float2 rx = make_float2(g0.x, g1.x), sx = make_float2(g0.y, g1.y);
  const float2 rz = make_float2(g0.z, g1.z), sz = make_float2(g0.w, g1.w);

  float2 X[NP], Z[NP], W[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    float2 drx = f2(0.f), dsx = f2(0.f), drz = f2(0.f), dsz = f2(0.f);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      drx = axpy_c(p2_dr(i * NP + n), vx[n], drx);
      drz = axpy_c(p2_dr(i * NP + n), vz[n], drz);
      dsx = axpy_c(p2_ds(i * NP + n), vx[n], dsx);
      dsz = axpy_c(p2_ds(i * NP + n), vz[n], dsz);
    }
    X[i] = fma2(rx, drx, mul2(sx, dsx));
    Z[i] = fma2(rz, drz, mul2(sz, dsz));
    W[i] = fma2(rx, drz, fma2(sx, dsz, fma2(rz, drx, mul2(sz, dsx))));
  }
#pragma unroll
  for (int j = 0; j < NF; j++) {
    float2 nx, nz;
    if (j == 0) { nx = mul2(f2(-0.5f), sx); nz = mul2(f2(-0.5f), sz); }
    else if (j == 1) { nx = mul2(f2(0.5f), add2(rx, sx)); nz = mul2(f2(0.5f), add2(rz, sz)); }
    else { nx = mul2(f2(-0.5f), rx); nz = mul2(f2(-0.5f), rz); }
    // the velocity fields carry no sponge factor in this pass: raw neighbour values
    const FaceLane a = face_lane(pick(f0, j)), b = face_lane(pick(f1, j));
    float2 px[NF], pz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      px[k] = gather_pair<FRESH>(m, a, b, 0, k);
      pz[k] = gather_pair<FRESH>(m, a, b, 6, k);
    }
    float2 fa[NF], fb[NF], fw[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const float2 dvx = sub2(px[k], vx[own]);
      const float2 dvz = sub2(pz[k], vz[own]);
      fa[k] = mul2(nx, dvx);
      fb[k] = mul2(nz, dvz);
      fw[k] = fma2(nz, dvx, mul2(nx, dvz));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const float l = p2_lift((j * NP + i) * NF + k);
        X[i] = axpy_c(l, fa[k], X[i]);
        Z[i] = axpy_c(l, fb[k], Z[i]);
        W[i] = axpy_c(l, fw[k], W[i]);
      }
  }
  const float4 m0 = __ldg(m.mat + e0), m1 = __ldg(m.mat + e1);
  const float dt = m.dt;
  const float2 dl2m = make_float2(dt * m0.w, dt * m1.w), dlam = make_float2(dt * m0.y, dt * m1.y);
  const float2 dmu = make_float2(dt * m0.z, dt * m1.z);
  const bool any_sponge = (f0.w | f1.w) & 1;
  float2 txx[NP], tzz[NP], txz[NP], cxx[NP], czz[NP], cxz[NP];
  float2* __restrict__ Cp = KAHAN ? reinterpret_cast<float2*>(m.C) + p : nullptr;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const float2 a = any_sponge ? __ldg(reinterpret_cast<const float2*>(m.sponge + (long long)i * m.Kp) + p) : f2(1.f);
    txx[i] = mul2(Up[(12 + i) * H], a);
    tzz[i] = mul2(Up[(18 + i) * H], a);
    txz[i] = mul2(Up[(24 + i) * H], a);
    if (KAHAN) {
      cxx[i] = mul2(Cp[(12 + i) * H], a); czz[i] = mul2(Cp[(18 + i) * H], a); cxz[i] = mul2(Cp[(24 + i) * H], a);
    }
  }
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const float2 dxx = fma2(dl2m, X[i], mul2(dlam, Z[i]));
    const float2 dzz = fma2(dlam, X[i], mul2(dl2m, Z[i]));
    const float2 dxz = mul2(dmu, W[i]);
    if (KAHAN) {
      kahan2(txx[i], cxx[i], dxx);
      kahan2(tzz[i], czz[i], dzz);
      kahan2(txz[i], cxz[i], dxz);
    } else {
      txx[i] = add2(txx[i], dxx);
      tzz[i] = add2(tzz[i], dzz);
      txz[i] = add2(txz[i], dxz);
    }
    Up[(12 + i) * H] = txx[i];
    Up[(18 + i) * H] = tzz[i];
    Up[(24 + i) * H] = txz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { Cp[(12 + i) * H] = cxx[i]; Cp[(18 + i) * H] = czz[i]; Cp[(24 + i) * H] = cxz[i]; }
  }
}

template <bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_stress_x2e(const __grid_constant__ Ops2 ops,
                                                       const __grid_constant__ MeshDev<float> m,
                                                       Counters* __restrict__ ctr) {
  pdl_enter();
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  const int lb = blockIdx.x + m.block0;
  if (lb >= m.n_elem_blocks) { record(m, lb - m.n_elem_blocks, t); return; }
  stress_x2e_body<KAHAN>(ops, m, lb, t);
}

}  // namespace dg
