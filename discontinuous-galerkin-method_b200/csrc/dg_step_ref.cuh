// dg_step_ref.cuh — bit-exact reference-operator step kernels (DG_FP64_REF).
#pragma once
#include "dg_common.cuh"

namespace dg {

// -------------------------------------------------------------------------------------------
// Reference-operator path (DG_FP64_REF): the reference's own per-element Dx, Dz, Q, A, B and its
// exact operation order, with every product and sum rounded separately (no FMA contraction).
// The only difference to OpenMP_Function.c is that a boundary face takes the exterior value +0
// where the reference forms T[0] * 0, which can differ in the sign of a zero.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// Row i of the element's Dx and Dz.  OTF: rebuilt from the element's (Rx, Sx, Rz, Sz) with the
// operations of Dx_Dz (fun_DG.c:1166-1190), each product and sum rounded on its own:
// dxd[i][k] = Rx Vr[i][k] + Sx Vs[i][k], then Dx[i][n] = sum over k = 0..5 of dxd[i][k] inv(V)[k][n]
// from 0 — the same doubles the reference stores (the host checks that at set-up).  Otherwise
// read from the caller's arrays.
template <bool OTF>
__device__ __forceinline__ void ref_rows(const Ops<double>& ops, const MeshDev<double>& m, int e, int i,
                                         double (&dx)[NP], double (&dz)[NP]) {
  if (OTF) {
    const double4 g = ld4(m.geo + e);  // Rx, Sx, Rz, Sz
    double ax[NP], az[NP];
#pragma unroll
    for (int k = 0; k < NP; k++) {
      ax[k] = add(mul(g.x, ops.Vr[i * NP + k]), mul(g.y, ops.Vs[i * NP + k]));
      az[k] = add(mul(g.z, ops.Vr[i * NP + k]), mul(g.w, ops.Vs[i * NP + k]));
    }
#pragma unroll
    for (int n = 0; n < NP; n++) {
      double fx = 0, fz = 0;
#pragma unroll
      for (int k = 0; k < NP; k++) {
        fx = add(fx, mul(ax[k], ops.Vi[k * NP + n]));
        fz = add(fz, mul(az[k], ops.Vi[k * NP + n]));
      }
      dx[n] = fx;
      dz[n] = fz;
    }
  } else {
#pragma unroll
    for (int n = 0; n < NP; n++) {
      dx[n] = __ldg(m.Dx + (i * NP + n) * (long long)m.Kp + e);
      dz[n] = __ldg(m.Dz + (i * NP + n) * (long long)m.Kp + e);
    }
  }
}

template <bool MULTI, bool OTF>
__global__ void __launch_bounds__(256) k_velocity_ref(const __grid_constant__ Ops<double> ops,
                                                      const __grid_constant__ MeshDev<double> one,
                                                      const MeshDev<double>* __restrict__ tab,
                                                      const int2* __restrict__ btab,
                                                      Counters* __restrict__ ctr) {
  pdl_enter();
  int lb;
  const MeshDev<double>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  const int S = m.S;
  const long long g = (long long)lb * blockDim.x + threadIdx.x;
  if (g >= (long long)m.K * S) return;
  int e, s;
  if (S == 1) { e = (int)g; s = 0; } else { e = (int)(g / S); s = (int)(g - (long long)e * S); }
  const long long P = m.P;
  const int Kp = m.Kp;
  double* Ug = m.U + g;
  double txx[NP], tzz[NP], txz[NP], vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    vx[i] = Ug[(0 + i) * P]; vz[i] = Ug[(6 + i) * P];
    txx[i] = Ug[(12 + i) * P]; tzz[i] = Ug[(18 + i) * P]; txz[i] = Ug[(24 + i) * P];
  }
  const int4 fc = __ldg(m.face + e);
  if (fc.w & 1) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const double a = __ldg(m.sponge + (long long)i * Kp + e);
      vx[i] = mul(vx[i], a); vz[i] = mul(vz[i], a);
      txx[i] = mul(txx[i], a); tzz[i] = mul(tzz[i], a); txz[i] = mul(txz[i], a);
    }
  }
  if (__ldg(m.src_elem + s) == e) {
    const double w = __ldg(m.wavelet + t);
#pragma unroll
    for (int i = 0; i < NP; i++) vz[i] = add(vz[i], mul(__ldg(m.src_fun + s * NP + i), w));
  }
  const double A0 = __ldg(m.AB + 0 * Kp + e), A1 = __ldg(m.AB + 1 * Kp + e);
  const double B0 = __ldg(m.AB + 5 * Kp + e), B1 = __ldg(m.AB + 6 * Kp + e);
  double abx[NP], abz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    double s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    double dxr[NP], dzr[NP];
    ref_rows<OTF>(ops, m, e, i, dxr, dzr);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      const double dx = dxr[n];
      const double dz = dzr[n];
      s1 = add(s1, mul(dx, txx[n]));
      s2 = add(s2, mul(dx, txz[n]));
      s3 = add(s3, mul(dz, tzz[n]));
      s4 = add(s4, mul(dz, txz[n]));
    }
    abx[i] = add(mul(A0, s1), mul(B0, s4));
    abz[i] = add(mul(A1, s2), mul(B1, s3));
  }
  double qx[NF][NP], qz[NF][NP];
  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    double pxx[NF], pzz[NF], pxz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { pxx[k] = 0.0; pzz[k] = 0.0; pxz[k] = 0.0; }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const double* Un = m.U + ((long long)nb * S + s);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        pxx[k] = Un[(12 + node) * P]; pzz[k] = Un[(18 + node) * P]; pxz[k] = Un[(24 + node) * P];
        if (code & 8) {
          const double a = __ldg(m.sponge + (long long)node * Kp + nb);
          pxx[k] = mul(pxx[k], a); pzz[k] = mul(pzz[k], a); pxz[k] = mul(pxz[k], a);
        }
      }
    }
    double jxx[NF], jzz[NF], jxz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      jxx[k] = sub(pxx[k], txx[own]); jzz[k] = sub(pzz[k], tzz[own]); jxz[k] = sub(pxz[k], txz[own]);
    }
    const double q0 = __ldg(m.Q + (j * 10 + 0) * (long long)Kp + e), q1 = __ldg(m.Q + (j * 10 + 1) * (long long)Kp + e);
    const double q2 = __ldg(m.Q + (j * 10 + 2) * (long long)Kp + e), q3 = __ldg(m.Q + (j * 10 + 3) * (long long)Kp + e);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      double lxx = 0, lzz = 0, lxz = 0;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const double l = ops.L[(j * NP + i) * NF + k];
        lxx = add(lxx, mul(l, jxx[k])); lzz = add(lzz, mul(l, jzz[k])); lxz = add(lxz, mul(l, jxz[k]));
      }
      qx[j][i] = add(mul(q0, lxx), mul(q1, lxz));
      qz[j][i] = add(mul(q2, lzz), mul(q3, lxz));
    }
  }
  const double dt = m.dt;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    Ug[(0 + i) * P] = add(mul(add(add(add(abx[i], qx[0][i]), qx[1][i]), qx[2][i]), dt), vx[i]);
    Ug[(6 + i) * P] = add(mul(add(add(add(abz[i], qz[0][i]), qz[1][i]), qz[2][i]), dt), vz[i]);
  }
}

template <bool MULTI, bool OTF>
__global__ void __launch_bounds__(256) k_stress_ref(const __grid_constant__ Ops<double> ops,
                                                    const __grid_constant__ MeshDev<double> one,
                                                    const MeshDev<double>* __restrict__ tab,
                                                    const int2* __restrict__ btab,
                                                    Counters* __restrict__ ctr) {
  pdl_enter();
  int lb;
  const MeshDev<double>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  if (lb >= m.n_elem_blocks) { record(m, lb - m.n_elem_blocks, t); return; }
  const int S = m.S;
  const long long g = (long long)lb * blockDim.x + threadIdx.x;
  if (g >= (long long)m.K * S) return;
  int e, s;
  if (S == 1) { e = (int)g; s = 0; } else { e = (int)(g / S); s = (int)(g - (long long)e * S); }
  const long long P = m.P;
  const int Kp = m.Kp;
  double* Ug = m.U + g;
  double vx[NP], vz[NP], txx[NP], tzz[NP], txz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    vx[i] = Ug[(0 + i) * P]; vz[i] = Ug[(6 + i) * P];
    txx[i] = Ug[(12 + i) * P]; tzz[i] = Ug[(18 + i) * P]; txz[i] = Ug[(24 + i) * P];
  }
  const int4 fc = __ldg(m.face + e);
  if (fc.w & 1) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const double a = __ldg(m.sponge + (long long)i * Kp + e);
      txx[i] = mul(txx[i], a); tzz[i] = mul(tzz[i], a); txz[i] = mul(txz[i], a);
    }
  }
  double A[5], B[5];
#pragma unroll
  for (int q = 0; q < 5; q++) { A[q] = __ldg(m.AB + q * Kp + e); B[q] = __ldg(m.AB + (5 + q) * Kp + e); }
  double abxx[NP], abzz[NP], abxz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    double s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    double dxr[NP], dzr[NP];
    ref_rows<OTF>(ops, m, e, i, dxr, dzr);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      const double dx = dxr[n];
      const double dz = dzr[n];
      s1 = add(s1, mul(dx, vx[n]));
      s2 = add(s2, mul(dx, vz[n]));
      s3 = add(s3, mul(dz, vx[n]));
      s4 = add(s4, mul(dz, vz[n]));
    }
    abxx[i] = add(mul(A[2], s1), mul(B[2], s4));
    abzz[i] = add(mul(A[3], s1), mul(B[3], s4));
    abxz[i] = add(mul(A[4], s2), mul(B[4], s3));
  }
  double fxx[NF][NP], fzz[NF][NP], fxz[NF][NP];
  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    double px[NF], pz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { px[k] = 0.0; pz[k] = 0.0; }
    } else {
      const int nb = code >> 4, nf = (code >> 1) & 3, flip = code & 1;
      const double* Un = m.U + ((long long)nb * S + s);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        px[k] = Un[(0 + node) * P]; pz[k] = Un[(6 + node) * P];
      }
    }
    double jx[NF], jz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      jx[k] = sub(px[k], vx[own]); jz[k] = sub(pz[k], vz[own]);
    }
    double q[6];
#pragma unroll
    for (int c = 0; c < 6; c++) q[c] = __ldg(m.Q + (j * 10 + 4 + c) * (long long)Kp + e);
#pragma unroll
    for (int i = 0; i < NP; i++) {
      double lx = 0, lz = 0;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const double l = ops.L[(j * NP + i) * NF + k];
        lx = add(lx, mul(l, jx[k])); lz = add(lz, mul(l, jz[k]));
      }
      fxx[j][i] = add(mul(q[0], lx), mul(q[1], lz));
      fzz[j][i] = add(mul(q[2], lx), mul(q[3], lz));
      fxz[j][i] = add(mul(q[4], lx), mul(q[5], lz));
    }
  }
  const double dt = m.dt;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    Ug[(12 + i) * P] = add(mul(add(add(add(abxx[i], fxx[0][i]), fxx[1][i]), fxx[2][i]), dt), txx[i]);
    Ug[(18 + i) * P] = add(mul(add(add(add(abzz[i], fzz[0][i]), fzz[1][i]), fzz[2][i]), dt), tzz[i]);
    Ug[(24 + i) * P] = add(mul(add(add(add(abxz[i], fxz[0][i]), fxz[1][i]), fxz[2][i]), dt), txz[i]);
  }
}

}  // namespace dg
