// dg_common.cuh — shared definitions of the sm_100a kernels of the DG elastic-wave time loop (P2, Np = 6, Nfp = 3).
//
// Data layout in HBM (one mesh):
//   state   30 planes, plane = 6*field + node (fields Vx, Vz, Txx, Tzz, Txz), element e in
//           locality order, shot s innermost, in one of two layouts (MeshDev::ES / PS give the
//           value (e, plane, s) at U[e*ES + plane*PS + s] for both):
//             plane-major   U[plane][e*S + s], plane stride P = Kp*S (kernel bodies with one
//                           (element, shot) or two elements per thread: a warp reads a plane as
//                           a contiguous run);
//             element-major U[e][plane][S] (the packed two-shot bodies: an element's 30 planes
//                           at compile-time offsets; a warp of S = 64 shots is one element).
//   geo     R4[Kp]  rx, sx, rz, sz (inverse Jacobian, as fun_DG.c:1162-1165)
//   mat     R4[Kp]  1/rho, lambda, mu, lambda + 2 mu (the distinct entries of A/B, fun_DG.c:1076-1086)
//   face    int4[Kp] three face codes and a flag word (see face_code below)
//   sponge  R[6][Kp] absorb_fun, read only for elements whose flag says they are in the sponge
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

// The P2 operators on the reference triangle for the node order of the reference's operator
// files (FeketeNew: (1,-1), (0,0), (-1,1), (0,-1), (-1,0), (-1,-1)).  Every entry is a multiple
// of 1/8: the files hold them to 8 digits, these are the exact values.  Dr = Vr inv(V) and
// Ds = Vs inv(V) each have 22 nonzeros of 36; p2_lift((j*6 + i)*3 + k) is S_j (face-j lift).  The packed
// FP32 bodies take their operators from here as compile-time constants (zeros skipped, +-1 as an
// add or a subtract); the host checks the operators it is given against them first.
__host__ __device__ constexpr float p2_dr(int q) {
  constexpr float v[36] = {1.5f,  0.f, 0.f, -2.f, 0.f,  0.5f,  0.5f, 1.f, 0.f, -1.f, -1.f, 0.5f,
                             -0.5f, 2.f, 0.f, 0.f,  -2.f, 0.5f,  0.5f, 0.f, 0.f, 0.f,  0.f,  -0.5f,
                             -0.5f, 1.f, 0.f, 1.f,  -1.f, -0.5f, -0.5f, 0.f, 0.f, 2.f, 0.f,  -1.5f};
  return v[q];
}
__host__ __device__ constexpr float p2_ds(int q) {
  constexpr float v[36] = {0.f, 2.f, -0.5f, -2.f, 0.f,  0.5f,  0.f, 1.f, 0.5f,  -1.f, -1.f, 0.5f,
                             0.f, 0.f, 1.5f,  0.f,  -2.f, 0.5f,  0.f, 1.f, -0.5f, -1.f, 1.f,  -0.5f,
                             0.f, 0.f, 0.5f,  0.f,  0.f,  -0.5f, 0.f, 0.f, -0.5f, 0.f,  2.f,  -1.5f};
  return v[q];
}
__host__ __device__ constexpr float p2_lift(int q) {
  constexpr float v[54] = {-0.5f,   2.f,   4.5f,   0.625f,  -1.5f, -0.625f, 1.f,    4.f,  1.f,
                               0.5f,    5.f,   0.5f,   -0.625f, -1.5f, 0.625f,  4.5f,   2.f,  -0.5f,
                               4.5f,    2.f,   -0.5f,  0.5f,    5.f,   0.5f,    -0.5f,  2.f,  4.5f,
                               -0.625f, -1.5f, 0.625f, 0.625f,  -1.5f, -0.625f, 1.f,    4.f,  1.f,
                               1.f,     4.f,   1.f,    0.625f,  -1.5f, -0.625f, -0.5f,  2.f,  4.5f,
                               -0.625f, -1.5f, 0.625f, 0.5f,    5.f,   0.5f,    4.5f,   2.f,  -0.5f};
  return v[q];
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
  // the parsed Vr, Vs, inv(V): the reference-operator path rebuilds Dx, Dz from them
  R Vr[NP * NP];
  R Vs[NP * NP];
  R Vi[NP * NP];
};

template <class R> struct MeshDev {
  long long P;            // plane stride of the plane-major layout (Kp * S)
  long long ES, PS;       // value (e, plane, s) lives at U[e*ES + plane*PS + s] in either layout
  long long steps;        // this mesh's wavelet length
  int K, Kp, S, n_rec;
  int n_elem_blocks;      // element blocks of this mesh (grid = these + recorder blocks)
  int block0;             // one-mesh launches: first element block of the launch, which covers
                          // blocks [block0, n_elem_blocks) and then the recorder blocks (a window
                          // of a split mesh's half step; 0 otherwise)
  int kind;               // FP32 kernel body: 0 one (element, shot) per thread, plane-major;
                          // 1 two elements per thread (S = 1); 2 two shots per thread, element-major
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

// Programmatic dependent launch (two-launch step kernels): wait until the previous kernel of the
// stream has completed and its stores are visible — at once when this launch did not ask to
// start early — then let the next kernel of the stream start its blocks, which wait the same way.
// The next kernel starts only once every block of this one has started, so no block waits for
// room that a waiting block holds.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// gpu-scope acquire load / release store of a flag, and a volatile load of an error word
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// a release pattern in two parts: the gpu-scope release fence, then a relaxed store of the flag
__device__ __forceinline__ void fence_release_gpu() { asm volatile("fence.release.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) { return *(volatile const int*)p; }

// 8 bytes from global to this thread's shared memory without a register (cp.async, through
// L1), the group commit, and the wait for this thread's copies
__device__ __forceinline__ void cp_async8(void* dst_smem, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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
  if (!MULTI) { local = blockIdx.x + one.block0; return &one; }
  const int2 b = __ldg(btab + blockIdx.x);
  local = b.y;
  return tab + b.x;
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


}  // namespace dg
