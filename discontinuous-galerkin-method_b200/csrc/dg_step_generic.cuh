// dg_step_generic.cuh — step kernels in the geometric-factor form for any shot count and for
// batches of meshes: FP64 and FP32 (plain or Kahan-compensated), one thread per (element, shot),
// plane-major layout U[plane][e*S + s].
//
// Register budget: the velocity kernel works in an x pass (Txx, Txz -> Vx) and a z pass
// (Txz, Tzz -> Vz), so only two stress fields are live at a time (the z pass gathers the
// neighbour's Txz a second time, from L1/L2); the stress kernel takes the volume terms first and
// the face terms after; the fields being updated are loaded only at the end.
#pragma once
#include "dg_common.cuh"

namespace dg {

// Outward normal of face j times |face| / (4 J) from the inverse Jacobian (rx, sx, rz, sz):
// (-sx,-sz)/2, (rx+sx,rz+sz)/2, (-rx,-rz)/2 — the reference's Q / A (fun_DG.c:1118-1131).
template <class R>
__device__ __forceinline__ void face_normal(int j, R rx, R sx, R rz, R sz, R& nx, R& nz) {
  if (j == 0) { nx = -sx * R(0.5); nz = -sz * R(0.5); }
  else if (j == 1) { nx = (rx + sx) * R(0.5); nz = (rz + sz) * R(0.5); }
  else { nx = -rx * R(0.5); nz = -rz * R(0.5); }
}

// The velocity right-hand side, both directions in one sweep over the faces:
//   hx = Dr (rx Txx + rz Txz) + Ds (sx Txx + sz Txz) + sum_j S_j (nx_j dTxx + nz_j dTxz)
//   hz = Dr (rx Txz + rz Tzz) + Ds (sx Txz + sz Tzz) + sum_j S_j (nz_j dTzz + nx_j dTxz)
// Neighbour values take the neighbour's sponge factor.  One sweep gathers each neighbour value
// once; in FP64 it also spills less than an x sweep and a z sweep (4 against 16 bytes at 128
// registers) and runs 16 % faster (388k-element slope: 42.5 against 50.9 us per launch).
template <class R>
__device__ __forceinline__ void velocity_rhs_both(const Ops<R>& ops, const MeshDev<R>& m, const int codes[3],
                                                  R rx, R sx, R rz, R sz, const R txx[NP], const R tzz[NP],
                                                  const R txz[NP], int s, R hx[NP], R hz[NP]) {
  const long long P = m.P;
#pragma unroll
  for (int i = 0; i < NP; i++) { hx[i] = R(0); hz[i] = R(0); }
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    R nx, nz;
    face_normal(j, rx, sx, rz, sz, nx, nz);
    R pxx[NF], pzz[NF], pxz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { pxx[k] = R(0); pzz[k] = R(0); pxz[k] = R(0); }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const R* __restrict__ Un = m.U + ((long long)nb * m.S + s);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        pxx[k] = Un[(12 + node) * P];
        pzz[k] = Un[(18 + node) * P];
        pxz[k] = Un[(24 + node) * P];
      }
      if (code & 8) {
#pragma unroll
        for (int k = 0; k < NF; k++) {
          const R a = ldg(m.sponge + (long long)face_node(nf, flip ? 2 - k : k) * m.Kp + nb);
          pxx[k] *= a; pzz[k] *= a; pxz[k] *= a;
        }
      }
    }
    R fx[NF], fz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const R dxx = pxx[k] - txx[own], dzz = pzz[k] - tzz[own], dxz = pxz[k] - txz[own];
      fx[k] = nx * dxx + nz * dxz;
      fz[k] = nz * dzz + nx * dxz;
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        hx[i] += ops.L[(j * NP + i) * NF + k] * fx[k];
        hz[i] += ops.L[(j * NP + i) * NF + k] * fz[k];
      }
  }
  R a[NP], b[NP], c[NP], d[NP];
#pragma unroll
  for (int n = 0; n < NP; n++) {
    a[n] = rx * txx[n] + rz * txz[n];
    b[n] = sx * txx[n] + sz * txz[n];
    c[n] = rx * txz[n] + rz * tzz[n];
    d[n] = sx * txz[n] + sz * tzz[n];
  }
#pragma unroll
  for (int i = 0; i < NP; i++)
#pragma unroll
    for (int n = 0; n < NP; n++) {
      hx[i] += ops.Dr[i * NP + n] * a[n] + ops.Ds[i * NP + n] * b[n];
      hz[i] += ops.Dr[i * NP + n] * c[n] + ops.Ds[i * NP + n] * d[n];
    }
}

// Velocity half-step: for its own element the sponge on the five fields and the source on Vz
// (OpenMP_Function.c:25-58), then V += dt L_V(T) (OpenMP_Function.c:75-185), L_V = (1/rho) h.
template <class R, bool KAHAN>
__device__ __forceinline__ void velocity_body(const Ops<R>& ops, const MeshDev<R>& m, int lb, long long t) {
  const int S = m.S;
  const long long g = (long long)lb * blockDim.x + threadIdx.x;
  if (g >= (long long)m.K * S) return;
  int e, s;
  if (S == 1) { e = (int)g; s = 0; } else { e = (int)(g / S); s = (int)(g - (long long)e * S); }
  const long long P = m.P;
  R* __restrict__ Ug = m.U + g;

  const int4 fc = __ldg(m.face + e);
  const auto gm = ld4(m.geo + e);
  const R rx = gm.x, sx = gm.y, rz = gm.z, sz = gm.w;
  const bool own_sponge = fc.w & 1;
  const int codes[3] = {fc.x, fc.y, fc.z};
  R sp[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) sp[i] = own_sponge ? ldg(m.sponge + (long long)i * m.Kp + e) : R(1);

  R txz[NP], hx[NP], hz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) txz[i] = Ug[(24 + i) * P] * sp[i];
  {
    R txx[NP], tzz[NP];
#pragma unroll
    for (int i = 0; i < NP; i++) { txx[i] = Ug[(12 + i) * P] * sp[i]; tzz[i] = Ug[(18 + i) * P] * sp[i]; }
    velocity_rhs_both<R>(ops, m, codes, rx, sx, rz, sz, txx, tzz, txz, s, hx, hz);
  }

  const R irho = __ldg(&m.mat[e].x);
  R vx[NP], vz[NP], cvx[NP], cvz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = Ug[(0 + i) * P] * sp[i]; vz[i] = Ug[(6 + i) * P] * sp[i]; }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { cvx[i] = m.C[(0 + i) * P + g] * sp[i]; cvz[i] = m.C[(6 + i) * P + g] * sp[i]; }
  }
  R srcz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) srcz[i] = R(0);
  if (__ldg(m.src_elem + s) == e) {
    const R w = (R)__ldg(m.wavelet + t);
#pragma unroll
    for (int i = 0; i < NP; i++) srcz[i] = ldg(m.src_fun + s * NP + i) * w;
  }
  const R step = m.dt * irho;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const R dvx = step * hx[i];
    const R dvz = step * hz[i] + srcz[i];
    if (KAHAN) {
      R y = dvx - cvx[i];
      R tt = vx[i] + y;
      cvx[i] = (tt - vx[i]) - y;
      vx[i] = tt;
      y = dvz - cvz[i];
      tt = vz[i] + y;
      cvz[i] = (tt - vz[i]) - y;
      vz[i] = tt;
    } else {
      vx[i] += dvx;
      vz[i] += dvz;
    }
    Ug[(0 + i) * P] = vx[i];
    Ug[(6 + i) * P] = vz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { m.C[(0 + i) * P + g] = cvx[i]; m.C[(6 + i) * P + g] = cvz[i]; }
  }
}

template <class R, bool KAHAN, bool MULTI>
__global__ void __launch_bounds__(256, 2) k_velocity(const __grid_constant__ Ops<R> ops,
                                                     const __grid_constant__ MeshDev<R> one,
                                                     const MeshDev<R>* __restrict__ tab,
                                                     const int2* __restrict__ btab,
                                                     Counters* __restrict__ ctr) {
  pdl_enter();
  int lb;
  const MeshDev<R>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  velocity_body<R, KAHAN>(ops, m, lb, t);
}

// Stress half-step: T = a T + dt L_T(V) (OpenMP_Function.c:188-306),
//   Txx += dt [ (l+2m) (dxVx + sum_j S_j nx_j dVx) + l (dzVz + sum_j S_j nz_j dVz) ]
//   Tzz += dt [ l (dxVx + ...) + (l+2m) (dzVz + ...) ]
//   Txz += dt m [ dxVz + dzVx + sum_j S_j (nz_j dVx + nx_j dVz) ]
// The trailing blocks of the grid record the receivers (V is final during this kernel).
template <class R, bool KAHAN>
__device__ __forceinline__ void stress_body(const Ops<R>& ops, const MeshDev<R>& m, int lb, long long t) {
  const int S = m.S;
  const long long g = (long long)lb * blockDim.x + threadIdx.x;
  if (g >= (long long)m.K * S) return;
  int e, s;
  if (S == 1) { e = (int)g; s = 0; } else { e = (int)(g / S); s = (int)(g - (long long)e * S); }
  const long long P = m.P;
  R* __restrict__ Ug = m.U + g;

  R vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = Ug[(0 + i) * P]; vz[i] = Ug[(6 + i) * P]; }
  const int4 fc = __ldg(m.face + e);
  const auto gm = ld4(m.geo + e);
  const R rx = gm.x, sx = gm.y, rz = gm.z, sz = gm.w;

  R X[NP], Z[NP], W[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    R drx = R(0), dsx = R(0), drz = R(0), dsz = R(0);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      drx += ops.Dr[i * NP + n] * vx[n];
      dsx += ops.Ds[i * NP + n] * vx[n];
      drz += ops.Dr[i * NP + n] * vz[n];
      dsz += ops.Ds[i * NP + n] * vz[n];
    }
    X[i] = rx * drx + sx * dsx;
    Z[i] = rz * drz + sz * dsz;
    W[i] = rx * drz + sx * dsz + rz * drx + sz * dsx;
  }

  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    R nxj, nzj;
    face_normal(j, rx, sx, rz, sz, nxj, nzj);
    R px[NF], pz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { px[k] = R(0); pz[k] = R(0); }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const R* __restrict__ Un = m.U + ((long long)nb * S + s);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        px[k] = Un[(0 + node) * P];
        pz[k] = Un[(6 + node) * P];
      }
    }
    R fa[NF], fb[NF], fw[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const R dvx = px[k] - vx[own];
      const R dvz = pz[k] - vz[own];
      fa[k] = nxj * dvx;
      fb[k] = nzj * dvz;
      fw[k] = nzj * dvx + nxj * dvz;
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const R l = ops.L[(j * NP + i) * NF + k];
        X[i] += l * fa[k];
        Z[i] += l * fb[k];
        W[i] += l * fw[k];
      }
  }

  const auto mt = ld4(m.mat + e);
  const R lam = mt.y, mu = mt.z, l2m = mt.w;
  R txx[NP], tzz[NP], txz[NP], cxx[NP], czz[NP], cxz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    txx[i] = Ug[(12 + i) * P];
    tzz[i] = Ug[(18 + i) * P];
    txz[i] = Ug[(24 + i) * P];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      cxx[i] = m.C[(12 + i) * P + g]; czz[i] = m.C[(18 + i) * P + g]; cxz[i] = m.C[(24 + i) * P + g];
    }
  }
  if (fc.w & 1) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const R a = ldg(m.sponge + (long long)i * m.Kp + e);
      txx[i] *= a; tzz[i] *= a; txz[i] *= a;
      if (KAHAN) { cxx[i] *= a; czz[i] *= a; cxz[i] *= a; }
    }
  }
  const R dt = m.dt;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const R dxx = dt * (l2m * X[i] + lam * Z[i]);
    const R dzz = dt * (lam * X[i] + l2m * Z[i]);
    const R dxz = dt * (mu * W[i]);
    if (KAHAN) {
      R y = dxx - cxx[i]; R tt = txx[i] + y; cxx[i] = (tt - txx[i]) - y; txx[i] = tt;
      y = dzz - czz[i]; tt = tzz[i] + y; czz[i] = (tt - tzz[i]) - y; tzz[i] = tt;
      y = dxz - cxz[i]; tt = txz[i] + y; cxz[i] = (tt - txz[i]) - y; txz[i] = tt;
    } else {
      txx[i] += dxx;
      tzz[i] += dzz;
      txz[i] += dxz;
    }
    Ug[(12 + i) * P] = txx[i];
    Ug[(18 + i) * P] = tzz[i];
    Ug[(24 + i) * P] = txz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      m.C[(12 + i) * P + g] = cxx[i]; m.C[(18 + i) * P + g] = czz[i]; m.C[(24 + i) * P + g] = cxz[i];
    }
  }
}

template <class R, bool KAHAN, bool MULTI>
__global__ void __launch_bounds__(256, 2) k_stress(const __grid_constant__ Ops<R> ops,
                                                   const __grid_constant__ MeshDev<R> one,
                                                   const MeshDev<R>* __restrict__ tab,
                                                   const int2* __restrict__ btab,
                                                   Counters* __restrict__ ctr) {
  pdl_enter();
  int lb;
  const MeshDev<R>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  if (lb >= m.n_elem_blocks) { record(m, lb - m.n_elem_blocks, t); return; }
  stress_body<R, KAHAN>(ops, m, lb, t);
}

}  // namespace dg
