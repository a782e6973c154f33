// dg_kernels.cuh — sm_100a kernels of the DG elastic-wave time loop (P2, Np = 6, Nfp = 3).
//
// Data layout in HBM (one mesh):
//   state   U[plane][g], plane = 6*field + node (fields Vx, Vz, Txx, Tzz, Txz), g = e*S + s
//           (element e in locality order, shot s innermost); plane stride P = Kp*S.
//   geo     R4[Kp]  rx, sx, rz, sz (inverse Jacobian, as fun_DG.c:1162-1165)
//   mat     R4[Kp]  1/rho, lambda, mu, lambda + 2 mu (the distinct entries of A/B, fun_DG.c:1076-1086)
//   face    int4[Kp] three face codes and a flag word (see face_code below)
//   sponge  R[6][Kp] absorb_fun, read only for elements whose flag says they are in the sponge
// One thread advances one (element, shot) pair; a warp therefore reads every state plane as a
// contiguous run of 32 values, and for S >= 32 a neighbour gather is a contiguous run as well.
//
// Face code: -1 on the outer boundary (exterior state 0, Edge_flag = 0, fun_DG.c:720-738),
// else nb << 4 | nb_in_sponge << 3 | nb_face << 1 | flip, where nb is the neighbour element,
// nb_face its face that touches ours and flip says its face nodes run the other way
// (NeighborNodes, fun_DG.c:1195-1276).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dg {

constexpr int NP = 6;
constexpr int NF = 3;
constexpr int NPLANES = 30;

// P2 face nodes, 0-based, face j position k (IBE for N = 2, fun_DG.c:1046-1057):
// {5,3,0}, {0,1,2}, {5,4,2}, packed as nibbles so a runtime (face, k) needs no memory.
constexpr unsigned long long FACE_NODES = 0x245210035ULL;
__host__ __device__ __forceinline__ int face_node(int j, int k) {
  return (int)((FACE_NODES >> (4 * (3 * j + k))) & 15ULL);
}

template <class R> struct R4T;
template <> struct R4T<float> { using type = float4; };
template <> struct R4T<double> { using type = double4; };

// Constant operators, passed by value as kernel parameters so every FMA reads them straight
// from the parameter bank.  L[j][i][k] is the face-j lift (S_j of the reference).
template <class R> struct Ops {
  R Dr[NP * NP];
  R Ds[NP * NP];
  R L[NF * NP * NF];
  R M[NP * NP];  // reference mass matrix inv(V V^T), energy only
};

template <class R> struct MeshDev {
  long long P;            // plane stride of the plane-major layout (Kp * S)
  long long ES, PS;       // value (e, plane, s) lives at U[e*ES + plane*PS + s] in either layout
  long long steps;        // this mesh's wavelet length
  int K, Kp, S, n_rec;
  int n_elem_blocks;      // element blocks of this mesh (grid = these + recorder blocks)
  int sponge_elems;
  R dt;
  R* U;                   // [30][P]
  R* C;                   // Kahan compensation [30][P] (FP32_KAHAN) or null
  const typename R4T<R>::type* geo;
  const typename R4T<R>::type* mat;
  const int4* face;
  const R* sponge;        // [6][Kp]
  const double* wavelet;  // [steps]
  const int* src_elem;    // [S]
  const R* src_fun;       // [S][6]
  const int* rec_elem;    // [n_rec]
  const int* rec_node;    // [n_rec]
  R* trace;               // [steps][2][n_rec][S]
  // reference-operator (bit-exact) path
  const double* Dx;       // [36][Kp]
  const double* Dz;       // [36][Kp]
  const double* Q;        // [30][Kp]
  const double* AB;       // [10][Kp]: A0..A4, B0..B4
};

// step counters: ctr[0] is read by the velocity kernel, ctr[1] by the stress kernel.  Each
// kernel writes only the counter the other one reads, so a captured graph can be replayed.
struct Counters { long long v, s; };

template <class R> __device__ __forceinline__ R ldg(const R* p) { return __ldg(p); }
__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ld4(const double4* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// -------------------------------------------------------------------------------------------
// block -> (mesh, local block) for batches of several meshes
struct BlockMap { int mesh; int local; };

template <bool MULTI, class R>
__device__ __forceinline__ const MeshDev<R>* pick_mesh(const MeshDev<R>& one, const MeshDev<R>* tab,
                                                        const int2* btab, int& local) {
  if (!MULTI) { local = blockIdx.x; return &one; }
  const int2 b = __ldg(btab + blockIdx.x);
  local = b.y;
  return tab + b.x;
}

// -------------------------------------------------------------------------------------------
// Velocity half-step, geometric-factor form.  Applies, for its own element, the sponge to the
// five fields and the source to Vz (OpenMP_Function.c:25-58) and then V += dt L_V(T)
// (OpenMP_Function.c:75-185) with
//   L_Vx = (1/rho) [ Dr (rx Txx + rz Txz) + Ds (sx Txx + sz Txz) + sum_j S_j (nx_j dTxx + nz_j dTxz) ]
//   L_Vz = (1/rho) [ Dr (rx Txz + rz Tzz) + Ds (sx Txz + sz Tzz) + sum_j S_j (nz_j dTzz + nx_j dTxz) ]
// where (nx_j, nz_j) is the outward normal times |face| / (4 J), i.e. (-sx,-sz)/2, (rx+sx,rz+sz)/2,
// (-rx,-rz)/2 for faces 0, 1, 2 — the reference's Q / A (fun_DG.c:1118-1131).  Neighbour
// values entering the jumps get the neighbour's sponge factor, as the reference applies the
// sponge to every element before the velocity pass.
template <class R, bool KAHAN, bool MULTI>
__global__ void __launch_bounds__(256) k_velocity(const __grid_constant__ Ops<R> ops,
                                                  const __grid_constant__ MeshDev<R> one,
                                                  const MeshDev<R>* __restrict__ tab,
                                                  const int2* __restrict__ btab,
                                                  Counters* __restrict__ ctr) {
  int lb;
  const MeshDev<R>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
  const long long t = ctr->v;
  if (!MULTI || blockIdx.x == 0) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  }
  if (t >= m.steps) return;
  const int S = m.S;
  const long long g = (long long)lb * blockDim.x + threadIdx.x;
  if (g >= (long long)m.K * S) return;
  int e, s;
  if (S == 1) { e = (int)g; s = 0; } else { e = (int)(g / S); s = (int)(g - (long long)e * S); }
  const long long P = m.P;
  R* __restrict__ Ug = m.U + g;

  R txx[NP], tzz[NP], txz[NP], vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    vx[i] = Ug[(0 + i) * P];
    vz[i] = Ug[(6 + i) * P];
    txx[i] = Ug[(12 + i) * P];
    tzz[i] = Ug[(18 + i) * P];
    txz[i] = Ug[(24 + i) * P];
  }
  R cvx[NP], cvz[NP];
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { cvx[i] = m.C[(0 + i) * P + g]; cvz[i] = m.C[(6 + i) * P + g]; }
  }
  const int4 fc = __ldg(m.face + e);
  const auto gm = ld4(m.geo + e);
  const R rx = gm.x, sx = gm.y, rz = gm.z, sz = gm.w;
  const R irho = __ldg(&m.mat[e].x);

  if (fc.w & 1) {  // own element lies in the sponge
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const R a = ldg(m.sponge + (long long)i * m.Kp + e);
      txx[i] *= a; tzz[i] *= a; txz[i] *= a; vx[i] *= a; vz[i] *= a;
      if (KAHAN) { cvx[i] *= a; cvz[i] *= a; }
    }
  }
  R srcz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) srcz[i] = R(0);
  if (__ldg(m.src_elem + s) == e) {
    const R w = (R)__ldg(m.wavelet + t);
#pragma unroll
    for (int i = 0; i < NP; i++) srcz[i] = ldg(m.src_fun + s * NP + i) * w;
  }

  // volume terms
  R hx[NP], hz[NP];
  {
    R ax[NP], bx[NP], az[NP], bz[NP];
#pragma unroll
    for (int n = 0; n < NP; n++) {
      ax[n] = rx * txx[n] + rz * txz[n];
      bx[n] = sx * txx[n] + sz * txz[n];
      az[n] = rx * txz[n] + rz * tzz[n];
      bz[n] = sx * txz[n] + sz * tzz[n];
    }
#pragma unroll
    for (int i = 0; i < NP; i++) {
      R a = R(0), b = R(0);
#pragma unroll
      for (int n = 0; n < NP; n++) {
        a += ops.Dr[i * NP + n] * ax[n] + ops.Ds[i * NP + n] * bx[n];
        b += ops.Dr[i * NP + n] * az[n] + ops.Ds[i * NP + n] * bz[n];
      }
      hx[i] = a;
      hz[i] = b;
    }
  }

  // surface terms
  const int codes[3] = {fc.x, fc.y, fc.z};
#pragma unroll
  for (int j = 0; j < NF; j++) {
    const int code = codes[j];
    R nxj, nzj;
    if (j == 0) { nxj = -sx * R(0.5); nzj = -sz * R(0.5); }
    else if (j == 1) { nxj = (rx + sx) * R(0.5); nzj = (rz + sz) * R(0.5); }
    else { nxj = -rx * R(0.5); nzj = -rz * R(0.5); }
    R pxx[NF], pzz[NF], pxz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { pxx[k] = R(0); pzz[k] = R(0); pxz[k] = R(0); }
    } else {
      const int nb = code >> 4;
      const int nf = (code >> 1) & 3;
      const int flip = code & 1;
      const R* Un = m.U + ((long long)nb * S + s);
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
          const int node = face_node(nf, flip ? 2 - k : k);
          const R a = ldg(m.sponge + (long long)node * m.Kp + nb);
          pxx[k] *= a; pzz[k] *= a; pxz[k] *= a;
        }
      }
    }
    R fx[NF], fz[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const R dxx = pxx[k] - txx[own];
      const R dzz = pzz[k] - tzz[own];
      const R dxz = pxz[k] - txz[own];
      fx[k] = nxj * dxx + nzj * dxz;
      fz[k] = nzj * dzz + nxj * dxz;
    }
#pragma unroll
    for (int i = 0; i < NP; i++) {
#pragma unroll
      for (int k = 0; k < NF; k++) {
        hx[i] += ops.L[(j * NP + i) * NF + k] * fx[k];
        hz[i] += ops.L[(j * NP + i) * NF + k] * fz[k];
      }
    }
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

// Receiver gather of the reference's Record (OpenMP_Function.c:61-72, stride 2): thread q of
// the recorder blocks copies V at (receiver element, node) for one (receiver, shot).
template <class R>
__device__ __forceinline__ void record(const MeshDev<R>& m, int lb_rec, long long t) {
  const int q = lb_rec * blockDim.x + threadIdx.x;
  const int S = m.S;
  if (q >= m.n_rec * S) return;
  const int r = q / S, s = q - r * S;
  const int e = __ldg(m.rec_elem + r), node = __ldg(m.rec_node + r);
  const long long at = (long long)e * m.ES + s;
  R* tr = m.trace + (t * 2) * (long long)m.n_rec * S;
  tr[q] = m.U[at + (0 + node) * m.PS];
  tr[(long long)m.n_rec * S + q] = m.U[at + (6 + node) * m.PS];
}

// Stress half-step, geometric-factor form: T = a T + dt L_T(V) (OpenMP_Function.c:188-306),
//   Txx += dt [ (l+2m) (dxVx + sum_j S_j nx_j dVx) + l (dzVz + sum_j S_j nz_j dVz) ]
//   Tzz += dt [ l (dxVx + ...) + (l+2m) (dzVz + ...) ]
//   Txz += dt m [ dxVz + dzVx + sum_j S_j (nz_j dVx + nx_j dVz) ]
// The trailing blocks of the grid record the receivers (V is final during this kernel).
template <class R, bool KAHAN, bool MULTI>
__global__ void __launch_bounds__(256) k_stress(const __grid_constant__ Ops<R> ops,
                                                const __grid_constant__ MeshDev<R> one,
                                                const MeshDev<R>* __restrict__ tab,
                                                const int2* __restrict__ btab,
                                                Counters* __restrict__ ctr) {
  int lb;
  const MeshDev<R>& m = *pick_mesh<MULTI>(one, tab, btab, lb);
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
  R* __restrict__ Ug = m.U + g;

  R vx[NP], vz[NP], txx[NP], tzz[NP], txz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    vx[i] = Ug[(0 + i) * P];
    vz[i] = Ug[(6 + i) * P];
    txx[i] = Ug[(12 + i) * P];
    tzz[i] = Ug[(18 + i) * P];
    txz[i] = Ug[(24 + i) * P];
  }
  R cxx[NP], czz[NP], cxz[NP];
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      cxx[i] = m.C[(12 + i) * P + g]; czz[i] = m.C[(18 + i) * P + g]; cxz[i] = m.C[(24 + i) * P + g];
    }
  }
  const int4 fc = __ldg(m.face + e);
  const auto gm = ld4(m.geo + e);
  const R rx = gm.x, sx = gm.y, rz = gm.z, sz = gm.w;
  const auto mt = ld4(m.mat + e);
  const R lam = mt.y, mu = mt.z, l2m = mt.w;

  if (fc.w & 1) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      const R a = ldg(m.sponge + (long long)i * m.Kp + e);
      txx[i] *= a; tzz[i] *= a; txz[i] *= a;
      if (KAHAN) { cxx[i] *= a; czz[i] *= a; cxz[i] *= a; }
    }
  }

  // volume: X = dxVx, Z = dzVz, W = dxVz + dzVx
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
    if (j == 0) { nxj = -sx * R(0.5); nzj = -sz * R(0.5); }
    else if (j == 1) { nxj = (rx + sx) * R(0.5); nzj = (rz + sz) * R(0.5); }
    else { nxj = -rx * R(0.5); nzj = -rz * R(0.5); }
    R px[NF], pz[NF];
    if (code < 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) { px[k] = R(0); pz[k] = R(0); }
    } else {
      const int nb = code >> 4;
      const int nf = (code >> 1) & 3;
      const int flip = code & 1;
      const R* Un = m.U + ((long long)nb * S + s);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        px[k] = Un[(0 + node) * P];
        pz[k] = Un[(6 + node) * P];
      }
    }
    R fa[NF], fb[NF], fcw[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int own = face_node(j, k);
      const R dvx = px[k] - vx[own];
      const R dvz = pz[k] - vz[own];
      fa[k] = nxj * dvx;
      fb[k] = nzj * dvz;
      fcw[k] = nzj * dvx + nxj * dvz;
    }
#pragma unroll
    for (int i = 0; i < NP; i++) {
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const R l = ops.L[(j * NP + i) * NF + k];
        X[i] += l * fa[k];
        Z[i] += l * fb[k];
        W[i] += l * fcw[k];
      }
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

// -------------------------------------------------------------------------------------------
// Reference-operator path (DG_FP64_REF): the reference's own per-element Dx, Dz, Q, A, B and its
// exact operation order, with every product and sum rounded separately (no FMA contraction).
// The only difference to OpenMP_Function.c is that a boundary face takes the exterior value +0
// where the reference forms T[0] * 0, which can differ in the sign of a zero.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

template <bool MULTI>
__global__ void __launch_bounds__(256) k_velocity_ref(const __grid_constant__ Ops<double> ops,
                                                      const __grid_constant__ MeshDev<double> one,
                                                      const MeshDev<double>* __restrict__ tab,
                                                      const int2* __restrict__ btab,
                                                      Counters* __restrict__ ctr) {
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
#pragma unroll
    for (int n = 0; n < NP; n++) {
      const double dx = __ldg(m.Dx + (i * NP + n) * (long long)Kp + e);
      const double dz = __ldg(m.Dz + (i * NP + n) * (long long)Kp + e);
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

template <bool MULTI>
__global__ void __launch_bounds__(256) k_stress_ref(const __grid_constant__ Ops<double> ops,
                                                    const __grid_constant__ MeshDev<double> one,
                                                    const MeshDev<double>* __restrict__ tab,
                                                    const int2* __restrict__ btab,
                                                    Counters* __restrict__ ctr) {
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
#pragma unroll
    for (int n = 0; n < NP; n++) {
      const double dx = __ldg(m.Dx + (i * NP + n) * (long long)Kp + e);
      const double dz = __ldg(m.Dz + (i * NP + n) * (long long)Kp + e);
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

// -------------------------------------------------------------------------------------------
// Two-shot FP32 kernels for even shot counts, on Blackwell's packed FP32x2 arithmetic
// (__ffma2_rn / __fmul2_rn / __fadd2_rn: one instruction advances two shots).  Layout:
// element-major with shots innermost, U[e][plane][S], so thread q of an element owns shots 2q and
// 2q+1 as one float2 and all 30 planes of its element sit at compile-time offsets (multiples of
// S/2 float2) from one base address; a neighbour's planes likewise from nb * 30 * S/2.  The
// operator constants come pre-duplicated as float2 pairs so they feed the packed FMAs directly.
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

// Kahan-compensated u += d with compensation c (both lanes)
__device__ __forceinline__ void kahan2(float2& u, float2& c, float2 d) {
  const float2 y = sub2(d, c);
  const float2 t = add2(u, y);
  c = sub2(sub2(t, u), y);
  u = t;
}

template <int S, bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_velocity_x2(const __grid_constant__ Ops2 ops,
                                                        const __grid_constant__ MeshDev<float> m,
                                                        Counters* __restrict__ ctr) {
  constexpr int H = S / 2;    // float2 lanes per element
  constexpr int ES = 30 * H;  // element stride in float2
  const long long t = ctr->v;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->s = t;
  if (t >= m.steps) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m.K * H) return;
  const int e = g / H, q = g - e * H;
  float2* __restrict__ Ue = reinterpret_cast<float2*>(m.U) + (long long)e * ES + q;

  float2 txx[NP], tzz[NP], txz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    txx[i] = Ue[(12 + i) * H];
    tzz[i] = Ue[(18 + i) * H];
    txz[i] = Ue[(24 + i) * H];
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
      const float2* __restrict__ Un = reinterpret_cast<const float2*>(m.U) + (long long)nb * ES + q;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        pxx[k] = Un[(12 + node) * H];
        pzz[k] = Un[(18 + node) * H];
        pxz[k] = Un[(24 + node) * H];
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
        hx[i] = fma2(ops.L[(j * NP + i) * NF + k], fx[k], hx[i]);
        hz[i] = fma2(ops.L[(j * NP + i) * NF + k], fz[k], hz[i]);
      }
  }

  // volume terms: Dr (rx Txx + rz Txz) + Ds (sx Txx + sz Txz) and the same for (Txz, Tzz)
  const float2 rx = f2(gm.x), sx = f2(gm.y), rz = f2(gm.z), sz = f2(gm.w);
  {
    float2 a[NP], b[NP];
#pragma unroll
    for (int n = 0; n < NP; n++) {
      a[n] = fma2(rx, txx[n], mul2(rz, txz[n]));
      b[n] = fma2(sx, txx[n], mul2(sz, txz[n]));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int n = 0; n < NP; n++) {
        hx[i] = fma2(ops.Dr[i * NP + n], a[n], hx[i]);
        hx[i] = fma2(ops.Ds[i * NP + n], b[n], hx[i]);
      }
  }
  {
    float2 a[NP], b[NP];
#pragma unroll
    for (int n = 0; n < NP; n++) {
      a[n] = fma2(rx, txz[n], mul2(rz, tzz[n]));
      b[n] = fma2(sx, txz[n], mul2(sz, tzz[n]));
    }
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
      for (int n = 0; n < NP; n++) {
        hz[i] = fma2(ops.Dr[i * NP + n], a[n], hz[i]);
        hz[i] = fma2(ops.Ds[i * NP + n], b[n], hz[i]);
      }
  }

  // V = a V (+ source on Vz) + dt/rho * rhs
  float2 vx[NP], vz[NP], cx[NP], cz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = Ue[(0 + i) * H]; vz[i] = Ue[(6 + i) * H]; }
  float2* __restrict__ Ce = nullptr;
  if (KAHAN) {
    Ce = reinterpret_cast<float2*>(m.C) + (long long)e * ES + q;
#pragma unroll
    for (int i = 0; i < NP; i++) { cx[i] = Ce[(0 + i) * H]; cz[i] = Ce[(6 + i) * H]; }
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
    Ue[(0 + i) * H] = vx[i];
    Ue[(6 + i) * H] = vz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) { Ce[(0 + i) * H] = cx[i]; Ce[(6 + i) * H] = cz[i]; }
  }
}

template <int S, bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_stress_x2(const __grid_constant__ Ops2 ops,
                                                      const __grid_constant__ MeshDev<float> m,
                                                      Counters* __restrict__ ctr) {
  constexpr int H = S / 2;
  constexpr int ES = 30 * H;
  const long long t = ctr->s;
  if (threadIdx.x == 0 && blockIdx.x == 0) ctr->v = t + 1;
  if (t >= m.steps) return;
  if ((int)blockIdx.x >= m.n_elem_blocks) { record(m, blockIdx.x - m.n_elem_blocks, t); return; }
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m.K * H) return;
  const int e = g / H, q = g - e * H;
  float2* __restrict__ Ue = reinterpret_cast<float2*>(m.U) + (long long)e * ES + q;

  float2 vx[NP], vz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) { vx[i] = Ue[(0 + i) * H]; vz[i] = Ue[(6 + i) * H]; }
  const int4 fc = __ldg(m.face + e);
  const float4 gm = __ldg(m.geo + e);
  const float4 mt = __ldg(m.mat + e);
  const float2 rx = f2(gm.x), sx = f2(gm.y), rz = f2(gm.z), sz = f2(gm.w);

  // volume: X = dxVx, Z = dzVz, W = dxVz + dzVx
  float2 X[NP], Z[NP], W[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    float2 drx = f2(0.f), dsx = f2(0.f), drz = f2(0.f), dsz = f2(0.f);
#pragma unroll
    for (int n = 0; n < NP; n++) {
      drx = fma2(ops.Dr[i * NP + n], vx[n], drx);
      dsx = fma2(ops.Ds[i * NP + n], vx[n], dsx);
      drz = fma2(ops.Dr[i * NP + n], vz[n], drz);
      dsz = fma2(ops.Ds[i * NP + n], vz[n], dsz);
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
      const float2* __restrict__ Un = reinterpret_cast<const float2*>(m.U) + (long long)nb * ES + q;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const int node = face_node(nf, flip ? 2 - k : k);
        px[k] = Un[(0 + node) * H];
        pz[k] = Un[(6 + node) * H];
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
        const float2 l = ops.L[(j * NP + i) * NF + k];
        X[i] = fma2(l, fa[k], X[i]);
        Z[i] = fma2(l, fb[k], Z[i]);
        W[i] = fma2(l, fw[k], W[i]);
      }
  }

  float2 txx[NP], tzz[NP], txz[NP], cxx[NP], czz[NP], cxz[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    txx[i] = Ue[(12 + i) * H];
    tzz[i] = Ue[(18 + i) * H];
    txz[i] = Ue[(24 + i) * H];
  }
  float2* __restrict__ Ce = nullptr;
  if (KAHAN) {
    Ce = reinterpret_cast<float2*>(m.C) + (long long)e * ES + q;
#pragma unroll
    for (int i = 0; i < NP; i++) { cxx[i] = Ce[(12 + i) * H]; czz[i] = Ce[(18 + i) * H]; cxz[i] = Ce[(24 + i) * H]; }
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
    Ue[(12 + i) * H] = txx[i];
    Ue[(18 + i) * H] = tzz[i];
    Ue[(24 + i) * H] = txz[i];
  }
  if (KAHAN) {
#pragma unroll
    for (int i = 0; i < NP; i++) {
      Ce[(12 + i) * H] = cxx[i]; Ce[(18 + i) * H] = czz[i]; Ce[(24 + i) * H] = cxz[i];
    }
  }
}

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

// traces of steps [t0, t0+n) of every shot -> out[comp][s][t - t0][r]
template <class R>
__global__ void k_fetch_traces(const R* __restrict__ tr, int n_rec, int S, long long t0, long long n,
                               double* __restrict__ out) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = n * n_rec * S;
  if (q >= 2 * per) return;
  const int comp = (int)(q / per);
  long long rem = q - comp * per;
  const int s = (int)(rem / (n * n_rec));
  rem -= (long long)s * n * n_rec;
  const long long t = rem / n_rec;
  const int r = (int)(rem - t * n_rec);
  out[q] = (double)tr[(((t0 + t) * 2 + comp) * n_rec + r) * (long long)S + s];
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
