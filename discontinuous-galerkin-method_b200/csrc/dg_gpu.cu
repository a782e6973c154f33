// dg_gpu.cu — host side of the sm_100a DG engine: the C ABI of include/dg_gpu.h.
//
// dg_gpu_init validates the reference's set-up arrays, renumbers elements (along a Hilbert curve
// of their centroids, or in reverse Cuthill-McKee order for the wavefront step), converts the
// index maps into compact face codes and the per-element operators into geometric factors (or
// keeps the reference's own operators for DG_FP64_REF), chooses the kernel family and block
// size, builds the wavefront schedule where it applies, and uploads everything.  dg_gpu_step
// replays a CUDA graph of `graph_steps` steps; a step is one velocity and one stress launch (the
// stress launch also records the receivers) or one wavefront launch.  Further entry points:
// snapshots overlapped with stepping, half steps and halo copies for a mesh split over several
// contexts, the autotuner, checkpoint load/fetch, and the test hook of the wavefront waits.
#include "dg_gpu.h"
#include "dg_aux.cuh"
#include "dg_common.cuh"
#include "dg_kernels.cuh"

#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <vector>

using namespace dg;

namespace {

thread_local std::string g_last;

int cuda_fail(cudaError_t e, const char* what, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s (line %d): %s", what, line, cudaGetErrorString(e));
  g_last = buf;
  return e == cudaErrorMemoryAllocation ? DG_ERR_NOMEM : DG_ERR_CUDA;
}
#define CK(x)                                                \
  do {                                                       \
    cudaError_t e_ = (x);                                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, #x, __LINE__); \
  } while (0)

int fail(int code, const char* msg) {
  g_last = msg;
  return code;
}

// Hilbert index of (x, y) on a 2^16 grid (the classic rotate-and-accumulate walk).
uint64_t hilbert(uint32_t x, uint32_t y) {
  uint64_t d = 0;
  for (uint32_t s = 1u << 15; s > 0; s >>= 1) {
    uint32_t rx = (x & s) > 0, ry = (y & s) > 0;
    d += (uint64_t)s * s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) { x = s - 1 - (x & (s - 1)) + (x & ~(s - 1)); y = s - 1 - (y & (s - 1)) + (y & ~(s - 1)); }
      uint32_t t = x; x = y; y = t;
    }
  }
  return d;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

namespace dg {
void set_last_error(const char* msg) { g_last = msg ? msg : ""; }
}

struct MeshHostInfo {
  long K = 0;
  int Kp = 0, S = 0, n_rec = 0;
  int S_pad = 0;  // shots stored (S plus a silent shot where the packed kernels need an even count)
  int kind = 0;   // kernel body (MeshDev::kind)
  long steps = 0;
  std::vector<int> new_of_old;  // caller element -> internal element
  int* d_new_of_old = nullptr;
  double dt = 0;
  int elem_blocks = 0, rec_blocks = 0;
  long sponge_elems = 0;
};

struct dg_gpu_ctx {
  int device = 0;
  int precision = DG_FP64;
  bool is_double = true;
  bool kahan = false;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::vector<MeshHostInfo> mi;
  std::vector<MeshDev<double>> md_d;
  std::vector<MeshDev<float>> md_f;
  MeshDev<double>* d_tab_d = nullptr;
  MeshDev<float>* d_tab_f = nullptr;
  int2* d_btab_v = nullptr;
  int2* d_btab_t = nullptr;
  Counters* d_ctr = nullptr;
  double bytes_two_pass = 0, bytes_wave = 0;  // algorithmic bytes per step of the two step forms
  int* d_flag = nullptr;
  double* d_energy = nullptr;
  double* d_stage = nullptr;
  size_t stage_elems = 0;
  void* d_flush = nullptr;
  size_t flush_bytes = 0;
  Ops<double> ops_d{};
  Ops<float> ops_f{};
  Ops2 ops2{};
  // packed FP32x2 kernels in use: 0 none; 1 two elements per thread (one shot, plane-major
  // layout); S >= 2 two shots per thread (element-major layout U[e][plane][S])
  int x2 = 0;
  bool mx = false;  // FP32 batch of meshes: per-block dispatch to the packed bodies (k_*_mx)
  // the batch's steps in one persistent cooperative launch (k_step_mx_p) instead of two
  // launches a step; its grid, barrier words and error word
  bool mx_persistent = false;
  int blocks_mxp = 0;
  // two-launch step kernels start early (programmatic dependent launch), each waiting for the one
  // before it in `pdl_enter`: measured -1.6 % (388k one-shot mesh) to +1.6 % (200k, two shots),
  // so off unless DG_PDL=1
  bool pdl = false;
  // reference-operator path: Dx, Dz rebuilt in the kernels (one mesh, one shot, checked at set-up)
  bool ref_otf = false;
  unsigned mx_extra = 0, mx_spin = 1u << 22;  // barrier arrivals beyond the grid, poll limit
  unsigned* d_mxbar = nullptr;
  int* d_mxerr = nullptr;
  bool x2pm = false; // the two-shot bodies on the plane-major layout (MeshDev::kind 3)
  bool wave = false;  // one launch per step (k_step_wave / k_step_wave_p), RCM order, schedule in wv
  bool wave_persistent = false;  // k_step_wave_p: resident blocks looping over the tickets
  bool wave_async = false;       // ... with the old values staged in shared memory by cp.async
  int margin_warps_per_sm = 10;  // lag margin of the wavefront step beyond the unit bandwidth
  int blocks_p = 0;              // its grid
  Wave wv{};
  int stall_unit = -1, stall_saved = 0;  // wait-list entry replaced by dg_gpu_debug_stall_wave
  // split meshes (dg_gpu_half_step / dg_gpu_halo_*): the velocity half of a step has run and its
  // stress half has not; per mesh the internal elements sent to and received from other parts
  bool half_pending = false;
  struct Halo {
    int* d_send = nullptr;
    int* d_recv = nullptr;
    long n_send = 0, n_recv = 0;
  };
  // a half step run in two parts (dg_gpu_half_step_part): the parts of the open half that have
  // run (bit 0 boundary, bit 1 interior; 0 = none open) and that half.  Mesh 0's elements up to
  // part_eB (internal numbering) hold every element with a ghost face neighbour, those up to
  // part_eO every element that is not a ghost (from the halo lists).
  int part_done = 0, part_half = 0;
  long part_eB = 0, part_eO = 0;
  std::vector<Halo> halo;
  std::vector<int4> face_h;    // face codes of mesh 0 (internal numbering), for the wavefront schedule
  std::vector<int> rec_elem_h; // receiver elements of mesh 0 (internal numbering)
  int num_sms = 148;
  int block = 256;
  int blocks_v = 0, blocks_t = 0;
  bool multi = false;
  int graph_steps = 100;
  cudaGraphExec_t graph = nullptr;
  // a second graph of graph_steps / 4 steps, for calls of fewer steps than a whole graph
  cudaGraphExec_t graph_small = nullptr;
  int graph_small_steps = 0;
  int graph_block = 0;
  long t = 0;
  long max_steps = 0;
  int watchdog_every = 0;
  dg_gpu_stats stats{};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // snapshot pipeline (dg_gpu_step_snapshots): two device slots and two pinned host slots, each
  // holding Vx and Vz of one snapshot, a copy stream and per-slot events
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t snap_conv[2] = {nullptr, nullptr}, snap_copy[2] = {nullptr, nullptr};
  double* snap_dev = nullptr;
  double* snap_host = nullptr;
  size_t snap_elems = 0;  // doubles per field and slot
  // step marks: an event recorded on the context stream after each dg_gpu_step(_async) call and
  // the step count it ends at, so a trace fetch on the copy stream waits for the steps that
  // wrote its window and no later ones
  struct StepMark {
    long t_end = -1;
    cudaEvent_t ev = nullptr;
  };
  static constexpr int kMarks = 4;
  StepMark marks[kMarks];
  int mark_next = 0;
  cudaEvent_t ev_fetch = nullptr, ev_wavelet = nullptr;

  ~dg_gpu_ctx() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph_small) cudaGraphExecDestroy(graph_small);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (int k = 0; k < 2; k++) {
      if (snap_conv[k]) cudaEventDestroy(snap_conv[k]);
      if (snap_copy[k]) cudaEventDestroy(snap_copy[k]);
    }
    for (auto& m : marks)
      if (m.ev) cudaEventDestroy(m.ev);
    if (ev_fetch) cudaEventDestroy(ev_fetch);
    if (ev_wavelet) cudaEventDestroy(ev_wavelet);
    if (snap_host) cudaFreeHost(snap_host);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (void* p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
  template <class T> int alloc(T** out, size_t count) {
    void* p = nullptr;
    if (count == 0) count = 1;
    CK(cudaMalloc(&p, count * sizeof(T)));
    allocs.push_back(p);
    *out = (T*)p;
    return DG_OK;
  }
  template <class T> int upload(T** out, const std::vector<T>& h) {
    int rc = alloc(out, h.size());
    if (rc) return rc;
    if (!h.empty()) CK(cudaMemcpyAsync(*out, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return DG_OK;
  }
  // free one buffer made by alloc/upload (after the stream has finished with it)
  void release(const void* p) {
    if (!p) return;
    for (size_t k = 0; k < allocs.size(); k++)
      if (allocs[k] == p) {
        cudaStreamSynchronize(stream);
        cudaFree(allocs[k]);
        allocs.erase(allocs.begin() + (long)k);
        return;
      }
  }
};

namespace {

constexpr long long P2_IBE[9] = {6, 4, 1, 1, 2, 3, 6, 5, 3};

// Per-mesh host preparation shared by both arithmetic types.
struct Prepared {
  long K;
  int Kp, S, n_rec;
  int S_pad = 0;  // shots stored and computed (S, or S + 1 silent shot for the packed kernels)
  int kind = 0;   // kernel body, as MeshDev::kind
  std::vector<int> order;       // internal -> caller element
  std::vector<int> new_of_old;  // caller -> internal
  std::vector<double> geo;      // [Kp][4] rx sx rz sz
  std::vector<double> mat;      // [Kp][4] 1/rho lambda mu lambda+2mu
  std::vector<int4> face;       // [Kp]
  std::vector<double> sponge;   // [6][Kp]
  std::vector<int> src_elem;
  std::vector<double> src_fun;  // [S][6]
  std::vector<int> rec_elem, rec_node;
  std::vector<double> Dx, Dz, Q, AB;  // SoA, reference path only
  bool ref_otf = false;  // reference path: Dx, Dz rebuilt in the kernels (then not stored)
  long sponge_elems = 0;
};

// Reverse Cuthill-McKee numbering of the element adjacency graph (faces with Edge_flag = 1):
// breadth-first from a pseudo-peripheral element of each connected part, neighbours taken in
// order of increasing degree, the whole sequence reversed.  Keeps every element's neighbours
// within a narrow band of numbers.
std::vector<int> rcm_order(const dg_gpu_mesh& m, long K) {
  auto nbr = [&](long e, int f) -> long {
    if (m.Edge_flag[e * 3 + f] != 1) return -1;
    const long n = m.Neighbor[e * 3 + f] - 1;
    return (n >= 0 && n < K && n != e) ? n : -1;
  };
  std::vector<int> deg(K, 0);
#pragma omp parallel for schedule(static)
  for (long e = 0; e < K; e++)
    for (int f = 0; f < 3; f++) deg[e] += nbr(e, f) >= 0;
  // every element's neighbours in visiting order (increasing degree, then number), -1 padded
  std::vector<int> nbt((size_t)K * 3);
#pragma omp parallel for schedule(static)
  for (long e = 0; e < K; e++) {
    int out[3] = {-1, -1, -1}, n = 0;
    for (int f = 0; f < 3; f++) {
      const long x = nbr(e, f);
      if (x >= 0) out[n++] = (int)x;
    }
    std::sort(out, out + n, [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
    for (int q = 0; q < 3; q++) nbt[e * 3 + q] = out[q];
  }
  std::vector<int> stamp(K, -1), queue(K);
  std::vector<char> placed(K, 0);
  std::vector<int> seq;
  seq.reserve(K);
  int pass = 0;
  auto sorted_nbrs = [&](long e, long out[3]) {
    int n = 0;
    for (int q = 0; q < 3 && nbt[e * 3 + q] >= 0; q++) out[n++] = nbt[e * 3 + q];
    return n;
  };
  for (long s0 = 0; s0 < K; s0++) {
    if (placed[s0]) continue;
    // two sweeps to a far element of minimum degree in the last level
    long start = s0;
    for (int sweep = 0; sweep < 2; sweep++) {
      ++pass;
      int head = 0, tail = 0;
      queue[tail++] = (int)start;
      stamp[start] = pass;
      int level_begin = 0;
      while (head < tail) {
        const int level_end = tail;
        level_begin = head;
        while (head < level_end) {
          const long e = queue[head++];
          long nb[3];
          const int n = sorted_nbrs(e, nb);
          for (int q = 0; q < n; q++)
            if (stamp[nb[q]] != pass) {
              stamp[nb[q]] = pass;
              queue[tail++] = (int)nb[q];
            }
        }
      }
      long best = queue[level_begin];
      for (int q = level_begin; q < tail; q++)
        if (deg[queue[q]] < deg[best]) best = queue[q];
      start = best;
    }
    int head = (int)seq.size();
    seq.push_back((int)start);
    placed[start] = 1;
    while (head < (int)seq.size()) {
      const long e = seq[head++];
      long nb[3];
      const int n = sorted_nbrs(e, nb);
      for (int q = 0; q < n; q++)
        if (!placed[nb[q]]) {
          placed[nb[q]] = 1;
          seq.push_back((int)nb[q]);
        }
    }
  }
  std::reverse(seq.begin(), seq.end());
  return seq;
}

int prepare(const dg_gpu_mesh& m, int precision, int reorder, Prepared& p, bool want_otf = false) {
  if (m.K <= 0 || m.K > (1L << 26)) return fail(DG_ERR_ARG, "K must be in [1, 2^26]");
  if (m.Np != 6 || m.Nfp != 3) return fail(DG_ERR_UNSUPPORTED, "only P2 (Np = 6, Nfp = 3) is supported");
  if (!m.Point || !m.Triangle || m.n_points <= 0 || !m.Vr || !m.Vs || !m.inverV || !m.S || !m.ibe || !m.Neighbor ||
      !m.Node_Neighbor || !m.Edge_flag || !m.A || !m.B || !m.absorb_fun || !m.wavelet || m.n_steps <= 0)
    return fail(DG_ERR_ARG, "missing mesh array");
  if (m.n_shots < 1 || !m.source || !m.fun) return fail(DG_ERR_ARG, "need at least one shot with source and fun");
  if (m.n_rec < 0 || (m.n_rec > 0 && !m.receiver)) return fail(DG_ERR_ARG, "bad receivers");
  if (!(m.dt > 0) || !std::isfinite(m.dt)) return fail(DG_ERR_ARG, "dt must be positive and finite");
  if (precision == DG_FP64_REF && (!m.Dx || !m.Dz || !m.Q))
    return fail(DG_ERR_ARG, "DG_FP64_REF needs the reference's Dx, Dz and Q");
  for (int q = 0; q < 9; q++)
    if (m.ibe[q] != P2_IBE[q]) return fail(DG_ERR_UNSUPPORTED, "ibe is not the P2 face table {6,4,1},{1,2,3},{6,5,3}");
  if ((long long)m.n_shots * m.K > (1LL << 31) - 1) return fail(DG_ERR_ARG, "K * n_shots too large");

  const long K = m.K;
  p.K = K;
  p.S = m.n_shots;
  p.n_rec = m.n_rec;
  p.Kp = (int)((K + 31) / 32 * 32);
  const int Kp = p.Kp;

  // The per-element loops below run on OpenMP threads.  A loop that finds invalid input records
  // the first offending element (in loop order) and, after the loop, that element is checked
  // again to report the error a sequential loop would have stopped at.

  // geometry per caller element, as Dx_Dz (fun_DG.c:1150-1165)
  std::vector<double> cx(K), cz(K), rxa(K * 4);
  auto geometry = [&](long e) -> int {
    double X[3], Z[3];
    for (int v = 0; v < 3; v++) {
      long pt = m.Triangle[e * 3 + v] - 1;
      if (pt < 0 || pt >= m.n_points) return fail(DG_ERR_MESH, "Triangle holds a vertex index out of range");
      X[v] = m.Point[pt * 2 + 0];
      Z[v] = m.Point[pt * 2 + 1];
    }
    const double Xr = (X[1] - X[0]) * 0.5, Zr = (Z[1] - Z[0]) * 0.5;
    const double Xs = (X[2] - X[0]) * 0.5, Zs = (Z[2] - Z[0]) * 0.5;
    const double J = Xr * Zs - Xs * Zr;
    if (!(J > 0) && precision != DG_FP64_REF)
      return fail(DG_ERR_ORIENTATION, "a triangle is not counter-clockwise (Jacobian <= 0)");
    rxa[e * 4 + 0] = Zs / J;
    rxa[e * 4 + 1] = -Zr / J;
    rxa[e * 4 + 2] = -Xs / J;
    rxa[e * 4 + 3] = Xr / J;
    cx[e] = (X[0] + X[1] + X[2]) / 3.0;
    cz[e] = (Z[0] + Z[1] + Z[2]) / 3.0;
    return DG_OK;
  };
  long bad = K;
#pragma omp parallel for schedule(static) reduction(min : bad)
  for (long e = 0; e < K; e++)
    if (geometry(e) != DG_OK) bad = std::min(bad, e);
  if (bad < K) return geometry(bad);

  // locality order: Hilbert curve of centroids (1), or reverse Cuthill-McKee (2) for the
  // wavefront step, which needs every element's neighbours close to it in the numbering
  p.order.resize(K);
  for (long e = 0; e < K; e++) p.order[e] = (int)e;
  if (reorder == 2) {
    p.order = rcm_order(m, K);
  } else if (reorder) {
    double x0 = cx[0], x1 = cx[0], z0 = cz[0], z1 = cz[0];
    for (long e = 0; e < K; e++) {
      x0 = std::min(x0, cx[e]); x1 = std::max(x1, cx[e]);
      z0 = std::min(z0, cz[e]); z1 = std::max(z1, cz[e]);
    }
    const double span = std::max(x1 - x0, z1 - z0) + 1e-300;
    // (Hilbert index < 2^32) << 32 | element: distinct keys, so any sort gives the same order
    std::vector<uint64_t> key(K);
#pragma omp parallel for schedule(static)
    for (long e = 0; e < K; e++) {
      uint32_t ix = (uint32_t)std::min(65535.0, std::floor((cx[e] - x0) / span * 65535.0));
      uint32_t iz = (uint32_t)std::min(65535.0, std::floor((cz[e] - z0) / span * 65535.0));
      key[e] = hilbert(ix, iz) << 32 | (uint64_t)e;
    }
    __gnu_parallel::sort(key.begin(), key.end());
#pragma omp parallel for schedule(static)
    for (long e = 0; e < K; e++) p.order[e] = (int)(key[e] & 0xffffffffu);
  }
  p.new_of_old.assign(K, 0);
#pragma omp parallel for schedule(static)
  for (long n = 0; n < K; n++) p.new_of_old[p.order[n]] = (int)n;

  // sponge flags
  std::vector<char> in_sponge(K, 0);
#pragma omp parallel for schedule(static)
  for (long e = 0; e < K; e++)
    for (int i = 0; i < 6; i++)
      if (m.absorb_fun[e * 6 + i] != 1.0) in_sponge[e] = 1;

  p.geo.assign((size_t)Kp * 4, 0.0);
  p.mat.assign((size_t)Kp * 4, 0.0);
  p.face.assign(Kp, make_int4(-1, -1, -1, 0));
  p.sponge.assign((size_t)6 * Kp, 1.0);
  auto element = [&](long n) -> int {
    const long e = p.order[n];
    for (int c = 0; c < 4; c++) p.geo[n * 4 + c] = rxa[e * 4 + c];
    const double* A = m.A + e * 5;
    const double* B = m.B + e * 5;
    if (precision != DG_FP64_REF) {
      // the geometric-factor form relies on Elastic_A_B's structure (fun_DG.c:1076-1086)
      if (!(A[0] == A[1] && A[0] == B[0] && A[0] == B[1] && A[2] == B[3] && A[3] == B[2] && A[4] == B[4]))
        return fail(DG_ERR_MESH, "A/B do not have the structure Elastic_A_B produces");
    }
    p.mat[n * 4 + 0] = A[0];
    p.mat[n * 4 + 1] = A[3];
    p.mat[n * 4 + 2] = A[4];
    p.mat[n * 4 + 3] = A[2];
    int codes[3];
    for (int f = 0; f < 3; f++) {
      const long flag = m.Edge_flag[e * 3 + f];
      const long nb = m.Neighbor[e * 3 + f] - 1;
      if (nb < 0 || nb >= K) return fail(DG_ERR_MESH, "Neighbor holds an index out of range");
      if (flag == 0) { codes[f] = -1; continue; }
      if (flag != 1) return fail(DG_ERR_MESH, "Edge_flag must be 0 or 1");
      const long* nn = m.Node_Neighbor + e * 9 + f * 3;
      int found = -1;
      for (int g = 0; g < 3 && found < 0; g++) {
        bool same = true, rev = true;
        for (int k = 0; k < 3; k++) {
          same &= nn[k] == P2_IBE[g * 3 + k];
          rev &= nn[k] == P2_IBE[g * 3 + 2 - k];
        }
        if (same) found = g * 2;
        else if (rev) found = g * 2 + 1;
      }
      if (found < 0) return fail(DG_ERR_MESH, "Node_Neighbor is not a P2 face of the neighbour");
      codes[f] = (p.new_of_old[nb] << 4) | (in_sponge[nb] ? 8 : 0) | ((found >> 1) << 1) | (found & 1);
    }
    p.face[n] = make_int4(codes[0], codes[1], codes[2], in_sponge[e] ? 1 : 0);
    if (in_sponge[e])
      for (int i = 0; i < 6; i++) p.sponge[(size_t)i * Kp + n] = m.absorb_fun[e * 6 + i];
    return DG_OK;
  };
  bad = K;
  long sponge_elems = 0;
#pragma omp parallel for schedule(static) reduction(min : bad) reduction(+ : sponge_elems)
  for (long n = 0; n < K; n++) {
    if (element(n) != DG_OK) bad = std::min(bad, n);
    sponge_elems += in_sponge[p.order[n]];
  }
  if (bad < K) return element(bad);
  p.sponge_elems = sponge_elems;
  // padded (silent) shots: no source element, zero source vector
  p.src_elem.assign(p.S_pad, -1);
  p.src_fun.assign((size_t)p.S_pad * 6, 0.0);
  for (int s = 0; s < p.S; s++) {
    const long tri = m.source[s * 2 + 0] - 1, node = m.source[s * 2 + 1] - 1;
    if (tri < 0 || tri >= K || node < 0 || node >= 6) return fail(DG_ERR_MESH, "source out of range");
    p.src_elem[s] = p.new_of_old[tri];
    for (int i = 0; i < 6; i++) p.src_fun[s * 6 + i] = m.fun[s * 6 + i];
  }
  p.rec_elem.resize(p.n_rec);
  p.rec_node.resize(p.n_rec);
  for (int r = 0; r < p.n_rec; r++) {
    const long tri = m.receiver[r * 2 + 0] - 1, node = m.receiver[r * 2 + 1] - 1;
    if (tri < 0 || tri >= K || node < 0 || node >= 6) return fail(DG_ERR_MESH, "receiver out of range");
    p.rec_elem[r] = p.new_of_old[tri];
    p.rec_node[r] = (int)node;
  }
  if (precision == DG_FP64_REF) {
    // Dx, Dz rebuilt in the kernels when, for every element, the operations of Dx_Dz
    // (fun_DG.c:1166-1190: dxd = Rx Vr + Sx Vs, then dxd inv(V), each product and sum rounded on
    // its own, as here) give exactly the caller's arrays from this element's Rx, Sx, Rz, Sz
    bool otf = want_otf;
    if (otf) {
      int differ = 0;
#pragma omp parallel for schedule(static) reduction(| : differ)
      for (long e = 0; e < K; e++) {
        if (differ) continue;
        const double* g = &rxa[e * 4];  // Rx, Sx, Rz, Sz
        for (int i = 0; i < 6 && !differ; i++) {
          double ax[6], az[6];
          for (int k = 0; k < 6; k++) {
            const double a1 = g[0] * m.Vr[i * 6 + k], a2 = g[1] * m.Vs[i * 6 + k];
            const double b1 = g[2] * m.Vr[i * 6 + k], b2 = g[3] * m.Vs[i * 6 + k];
            ax[k] = a1 + a2;
            az[k] = b1 + b2;
          }
          for (int q = 0; q < 6; q++) {
            double fx = 0, fz = 0;
            for (int k = 0; k < 6; k++) {
              const double px = ax[k] * m.inverV[k * 6 + q], pz = az[k] * m.inverV[k * 6 + q];
              fx = fx + px;
              fz = fz + pz;
            }
            differ |= memcmp(&fx, &m.Dx[e * 36 + i * 6 + q], sizeof(double)) != 0 ||
                      memcmp(&fz, &m.Dz[e * 36 + i * 6 + q], sizeof(double)) != 0;
          }
        }
      }
      otf = !differ;
    }
    p.ref_otf = otf;
    if (!otf) {
      p.Dx.assign((size_t)36 * Kp, 0.0);
      p.Dz.assign((size_t)36 * Kp, 0.0);
    }
    p.Q.assign((size_t)30 * Kp, 0.0);
    p.AB.assign((size_t)10 * Kp, 0.0);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < K; n++) {
      const long e = p.order[n];
      if (!otf)
        for (int q = 0; q < 36; q++) {
          p.Dx[(size_t)q * Kp + n] = m.Dx[e * 36 + q];
          p.Dz[(size_t)q * Kp + n] = m.Dz[e * 36 + q];
        }
      for (int q = 0; q < 30; q++) p.Q[(size_t)q * Kp + n] = m.Q[e * 30 + q];
      for (int q = 0; q < 5; q++) {
        p.AB[(size_t)q * Kp + n] = m.A[e * 5 + q];
        p.AB[(size_t)(5 + q) * Kp + n] = m.B[e * 5 + q];
      }
    }
  }
  return DG_OK;
}

template <class R> std::vector<R> cast(const std::vector<double>& v) { return std::vector<R>(v.begin(), v.end()); }

template <class R>
int upload_mesh(dg_gpu_ctx* c, const dg_gpu_mesh& m, Prepared& p, MeshDev<R>& d) {
  using R4 = typename R4T<R>::type;
  int rc;
  memset(&d, 0, sizeof d);
  d.K = (int)p.K;
  d.Kp = p.Kp;
  d.S = p.S_pad;
  d.n_rec = p.n_rec;
  d.kind = p.kind;
  d.P = (long long)p.Kp * p.S_pad;
  if (p.kind == 2) {  // element-major: U[e][plane][S]
    d.ES = 30LL * p.S_pad;
    d.PS = p.S_pad;
  } else {            // plane-major: U[plane][e*S + s]
    d.ES = p.S_pad;
    d.PS = d.P;
  }
  d.steps = m.n_steps;
  d.dt = (R)m.dt;
  d.sponge_elems = (int)p.sponge_elems;
  if ((rc = c->alloc(&d.U, (size_t)NPLANES * d.P))) return rc;
  CK(cudaMemsetAsync(d.U, 0, sizeof(R) * NPLANES * d.P, c->stream));
  if (c->kahan) {
    if ((rc = c->alloc(&d.C, (size_t)NPLANES * d.P))) return rc;
    CK(cudaMemsetAsync(d.C, 0, sizeof(R) * NPLANES * d.P, c->stream));
  }
  std::vector<R4> geo(p.Kp), mat(p.Kp);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < p.Kp; n++) {
    geo[n] = {(R)p.geo[n * 4 + 0], (R)p.geo[n * 4 + 1], (R)p.geo[n * 4 + 2], (R)p.geo[n * 4 + 3]};
    mat[n] = {(R)p.mat[n * 4 + 0], (R)p.mat[n * 4 + 1], (R)p.mat[n * 4 + 2], (R)p.mat[n * 4 + 3]};
  }
  R4* g4;
  R4* m4;
  if ((rc = c->upload(&g4, geo))) return rc;
  if ((rc = c->upload(&m4, mat))) return rc;
  d.geo = g4;
  d.mat = m4;
  int4* f4;
  if ((rc = c->upload(&f4, p.face))) return rc;
  d.face = f4;
  R* sp;
  if ((rc = c->upload(&sp, cast<R>(p.sponge)))) return rc;
  d.sponge = sp;
  double* wv;
  if ((rc = c->upload(&wv, std::vector<double>(m.wavelet, m.wavelet + m.n_steps)))) return rc;
  d.wavelet = wv;
  int* se;
  if ((rc = c->upload(&se, p.src_elem))) return rc;
  d.src_elem = se;
  R* sf;
  if ((rc = c->upload(&sf, cast<R>(p.src_fun)))) return rc;
  d.src_fun = sf;
  int *re, *rn;
  if ((rc = c->upload(&re, p.rec_elem))) return rc;
  if ((rc = c->upload(&rn, p.rec_node))) return rc;
  d.rec_elem = re;
  d.rec_node = rn;
  const size_t trace_elems = (size_t)m.n_steps * 2 * std::max(1, p.n_rec) * p.S_pad;
  if ((rc = c->alloc(&d.trace, trace_elems))) return rc;
  CK(cudaMemsetAsync(d.trace, 0, sizeof(R) * trace_elems, c->stream));
  if (c->precision == DG_FP64_REF) {
    double *dx, *dz, *q, *ab;
    dx = dz = nullptr;  // absent when the kernels rebuild them
    if (!p.Dx.empty() && (rc = c->upload(&dx, p.Dx))) return rc;
    if (!p.Dz.empty() && (rc = c->upload(&dz, p.Dz))) return rc;
    if ((rc = c->upload(&q, p.Q))) return rc;
    if ((rc = c->upload(&ab, p.AB))) return rc;
    d.Dx = dx;
    d.Dz = dz;
    d.Q = q;
    d.AB = ab;
  }
  return DG_OK;
}

// True when the mesh's operators equal the compile-time P2 tables of the packed FP32 kernels:
// Dr = Vr inv(V), Ds = Vs inv(V) and the face lifts S_j, each entry to 1e-6 of the largest.
bool p2_operators_match(const dg_gpu_mesh& m) {
  double big = 0, err = 0;
  for (int i = 0; i < 6; i++)
    for (int q = 0; q < 6; q++) {
      double a = 0, b = 0;
      for (int k = 0; k < 6; k++) {
        a += m.Vr[i * 6 + k] * m.inverV[k * 6 + q];
        b += m.Vs[i * 6 + k] * m.inverV[k * 6 + q];
      }
      big = std::max(big, std::max(std::fabs(a), std::fabs(b)));
      err = std::max(err, std::max(std::fabs(a - p2_dr(i * 6 + q)), std::fabs(b - p2_ds(i * 6 + q))));
    }
  for (int q = 0; q < 54; q++) {
    big = std::max(big, std::fabs(m.S[q]));
    err = std::max(err, std::fabs(m.S[q] - p2_lift(q)));
  }
  return err <= 1e-6 * big;
}

template <class R> void fill_ops(Ops<R>& o, const dg_gpu_mesh& m) {
  // Dr = Vr inv(V), Ds = Vs inv(V) from the parsed operator files
  for (int i = 0; i < 6; i++)
    for (int q = 0; q < 6; q++) {
      double a = 0, b = 0;
      for (int k = 0; k < 6; k++) {
        a += m.Vr[i * 6 + k] * m.inverV[k * 6 + q];
        b += m.Vs[i * 6 + k] * m.inverV[k * 6 + q];
      }
      o.Dr[i * 6 + q] = (R)a;
      o.Ds[i * 6 + q] = (R)b;
    }
  for (int q = 0; q < 54; q++) o.L[q] = (R)m.S[q];
  for (int q = 0; q < 36; q++) {
    o.Vr[q] = (R)m.Vr[q];
    o.Vs[q] = (R)m.Vs[q];
    o.Vi[q] = (R)m.inverV[q];
  }
  // reference mass matrix inv(V V^T) = inverV^T inverV
  for (int i = 0; i < 6; i++)
    for (int k = 0; k < 6; k++) {
      double a = 0;
      for (int q = 0; q < 6; q++) a += m.inverV[q * 6 + i] * m.inverV[q * 6 + k];
      o.M[i * 6 + k] = (R)a;
    }
}

// grid and block tables for the current block size
template <class R> int layout(dg_gpu_ctx* c, std::vector<MeshDev<R>>& md, MeshDev<R>** d_tab) {
  const int B = c->block;
  std::vector<int2> bv, bt;
  for (size_t k = 0; k < md.size(); k++) {
    MeshHostInfo& h = c->mi[k];
    const long long lanes =
        h.kind == 1 ? h.Kp / 2 : (h.kind >= 2 ? (long long)h.K * (h.S_pad / 2) : (long long)h.K * h.S_pad);
    h.elem_blocks = (int)((lanes + B - 1) / B);
    h.rec_blocks = (h.n_rec * h.S_pad + B - 1) / B;
    md[k].n_elem_blocks = h.elem_blocks;
    for (int b = 0; b < h.elem_blocks; b++) bv.push_back(make_int2((int)k, b));
    for (int b = 0; b < h.elem_blocks + h.rec_blocks; b++) bt.push_back(make_int2((int)k, b));
  }
  c->blocks_v = (int)bv.size();
  c->blocks_t = (int)bt.size();
  if (c->multi) {
    if (!*d_tab) {
      int rc = c->alloc(d_tab, md.size());
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(*d_tab, md.data(), md.size() * sizeof(MeshDev<R>), cudaMemcpyHostToDevice, c->stream));
    // block tables are rebuilt for each block size; old ones stay allocated until free
    int rc = c->upload(&c->d_btab_v, bv);
    if (rc) return rc;
    rc = c->upload(&c->d_btab_t, bt);
    if (rc) return rc;
  }
  return DG_OK;
}

int wave_resident(dg_gpu_ctx* c, int& per_sm);

// dynamic shared memory of a wavefront launch: the staging slots of the async layout
size_t wave_smem(const dg_gpu_ctx* c) {
  if (!c->wave_persistent || !c->wave_async) return 0;
  const size_t slots = c->kahan ? wave_stage_slots<true>() : wave_stage_slots<false>();
  return (size_t)(c->block / 32) * slots * 32 * sizeof(float2);
}

// Sets the ticket counter to the step the counters hold, for a launch grid of G blocks.
__global__ void k_wave_sync(const Counters* __restrict__ ctr, unsigned long long* tickets, unsigned G) {
  *tickets = (unsigned long long)ctr->v * G;
}

// Schedule of the wavefront step for the current block size.  A unit is one warp's 32 threads of
// the element range (thread g works on element g / H, H = shots / 2); the wait list holds, per unit, the
// distinct units covering one of its elements or a neighbour of one; the lag L (in blocks) covers
// the unit bandwidth plus a margin of about 60 % of the resident warps, so a stress update
// seldom waits.  Receivers are listed under every unit that covers their element.
int build_wave(dg_gpu_ctx* c) {
  const MeshHostInfo& h = c->mi[0];
  // two-shot layout: H = S/2 threads per element; one-shot layout: thread p owns elements 2p and
  // 2p+1 of the Kp padded elements, so a warp covers 64 elements
  const bool one = c->x2 == 1;
  const long H = one ? 1 : h.S_pad / 2;
  if (c->block % 32) return fail(DG_ERR_UNSUPPORTED, "block size not a multiple of 32");
  const int WPB = c->block / 32;
  const long threads = one ? h.Kp / 2 : h.K * H;
  const long NUl = (threads + 31) / 32;
  if (NUl >= (1L << 30)) return fail(DG_ERR_UNSUPPORTED, "too many warps for the wavefront step");
  const int NU = (int)NUl, NB = (NU + WPB - 1) / WPB;
  auto first_unit = [&](long e) { return (int)(one ? e / 64 : e * H / 32); };
  auto last_unit = [&](long e) { return (int)(one ? e / 64 : ((e + 1) * H - 1) / 32); };
  std::vector<int> nstart(NU + 1, 0), nlist;
  nlist.reserve((size_t)NU * 6);
  int Lb = 0, W = 1;
  std::vector<int> tmp;
  for (int u = 0; u < NU; u++) {
    tmp.assign(1, u);  // a unit of padding elements only still lists itself
    const long e0 = one ? (long)u * 64 : (long)u * 32 / H;
    const long e1 = std::min<long>(h.K - 1, one ? (long)u * 64 + 63 : ((long)u * 32 + 31) / H);
    for (long e = e0; e <= e1; e++) {
      const int4 f = c->face_h[e];
      const long els[4] = {e, f.x >= 0 ? f.x >> 4 : -1, f.y >= 0 ? f.y >> 4 : -1, f.z >= 0 ? f.z >> 4 : -1};
      for (long x : els)
        if (x >= 0)
          for (int v = first_unit(x); v <= last_unit(x); v++) tmp.push_back(v);
    }
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    for (int k : tmp) nlist.push_back(k);
    nstart[u + 1] = (int)nlist.size();
    Lb = std::max(Lb, tmp.back() / WPB - u / WPB);
    W = std::max(W, (int)tmp.size());
  }
  if (W > 32) return fail(DG_ERR_UNSUPPORTED, "wavefront wait list longer than a warp");
  std::vector<int> wait((size_t)NU * W, -1);
  for (int u = 0; u < NU; u++)
    std::copy(nlist.begin() + nstart[u], nlist.begin() + nstart[u + 1], wait.begin() + (size_t)u * W);
  std::vector<int> rstart(NU + 1, 0), rlist;
  {
    std::vector<std::vector<int>> per(NU);
    for (int r = 0; r < h.n_rec; r++) {
      const long e = c->rec_elem_h[r];
      for (int v = first_unit(e); v <= last_unit(e); v++) per[v].push_back(r);
    }
    for (int u = 0; u < NU; u++) {
      rstart[u + 1] = rstart[u] + (int)per[u].size();
      rlist.insert(rlist.end(), per[u].begin(), per[u].end());
    }
    if (rlist.empty()) rlist.push_back(0);
  }
  // a new schedule for a new block size: the previous one's buffers are no longer needed
  c->release(c->wv.wait);
  c->release(c->wv.rec_start);
  c->release(c->wv.rec_list);
  c->release(c->wv.vflag);
  c->release(c->wv.tickets);
  c->release(c->wv.ptk);
  c->release(c->wv.error);
  c->wv = Wave{};
  int *d_wait, *d_rs, *d_rl;
  unsigned* d_flag;
  unsigned long long* d_tk;
  unsigned* d_ptk;
  int* d_err;
  int rc;
  if ((rc = c->upload(&d_wait, wait))) return rc;
  if ((rc = c->upload(&d_rs, rstart))) return rc;
  if ((rc = c->upload(&d_rl, rlist))) return rc;
  // flag NU is never published: dg_gpu_debug_stall_wave points a wait at it
  if ((rc = c->alloc(&d_flag, NU + 1))) return rc;
  if ((rc = c->alloc(&d_tk, 1))) return rc;
  if ((rc = c->alloc(&d_ptk, 2))) return rc;
  CK(cudaMemsetAsync(d_ptk, 0, sizeof(unsigned) * 2, c->stream));
  if ((rc = c->alloc(&d_err, 1))) return rc;
  CK(cudaMemsetAsync(d_flag, 0, sizeof(unsigned) * (NU + 1), c->stream));
  c->stall_unit = -1;
  CK(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
  Wave& w = c->wv;
  w.NU = NU;
  w.NB = NB;
  w.W = W;
  // margin over the bandwidth, in blocks: 10 warps per SM (about 60 % of the resident warps),
  // so that the velocity updates a stress update needs have mostly finished when it starts,
  // while the lag window stays in L2; measured flat from 1,200 to 1,800 warps on the 200k-element
  // batch, much slower below 1,000 (DG_WAVE_MARGIN overrides it, in blocks, for tuning)
  int margin = (c->num_sms * c->margin_warps_per_sm + WPB - 1) / WPB;
  if (const char* env = getenv("DG_WAVE_MARGIN")) margin = std::max(0, atoi(env));
  w.L = Lb + margin;
  w.wait = d_wait;
  w.vflag = d_flag;
  w.rec_start = d_rs;
  w.rec_list = d_rl;
  w.tickets = d_tk;
  w.ptk = d_ptk;
  w.error = d_err;
  w.spin_limit = 1u << 20;  // a million polls of an L2 line: well under a second
  c->blocks_v = NB + w.L;
  c->blocks_t = 0;
  w.inv_G = ~0ULL / (unsigned long long)c->blocks_v;
  if (c->wave_persistent) {
    int per_sm = 0;
    if ((rc = wave_resident(c, per_sm))) return rc;
    if (per_sm < 1) return fail(DG_ERR_UNSUPPORTED, "the persistent wavefront kernel does not fit an SM");
    c->blocks_p = std::min(c->blocks_v, per_sm * c->num_sms);
  }
  k_wave_sync<<<1, 1, 0, c->stream>>>(c->d_ctr, d_tk, (unsigned)c->blocks_v);
  CK(cudaGetLastError());
  return DG_OK;
}

// shot counts with a two-shot FP32 kernel instance (element-major), and with a plane-major one
bool x2_supported(int S) { return (S >= 2 && S <= 16 && S % 2 == 0) || S == 32 || S == 64 || S == 128; }
bool x2pm_supported(int S) { return S >= 2 && S <= 16 && S % 2 == 0; }

// Kernel body and stored shot count for a mesh of S shots: FP32 meshes use the packed bodies —
// two elements per thread for one shot, two shots per thread from two shots on (plane-major
// layout up to 14 stored shots, element-major above or for the wavefront step), an odd count
// padded with one silent shot — unless the caller asks for one (element, shot) per thread
// (variant 1).
void choose_kind(int S, long K, bool fp32, int variant, bool want_wave, int& kind, int& S_pad) {
  kind = 0;
  S_pad = S;
  if (!fp32 || variant == 1) return;
  if (S == 1) {
    kind = 1;
    return;
  }
  const int even = S + (S & 1);
  if (x2_supported(even) && (long long)K * (even / 2) < (1LL << 31)) {
    // plane-major packed body for 2..14 stored shots: the element-major one scatters a warp's
    // loads over a few element records (200k elements, two launches: 4 shots 333 G against
    // 269 G DOF-updates/s, 6: 357 against 284, 8: 382 against 358, 16: equal; at two shots it
    // gives each thread a whole element record, 163 G, below one (element, shot) per thread,
    // 248 G, while the plane-major body runs at 319 G, and 405 G against 276 G on 2M elements);
    // the wavefront step needs the element-major layout
    const bool pm = x2pm_supported(even) && (variant == 3 || (variant == 0 && !want_wave && even <= 14));
    kind = pm ? 3 : 2;
    S_pad = even;
  }
}

// A two-launch step kernel on the context stream, asking to start before the previous kernel
// ends (its blocks wait in pdl_enter until that kernel has finished)
template <typename... K, typename... A>
int launch_k(dg_gpu_ctx* c, void (*kernel)(K...), dim3 grid, dim3 block, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = c->pdl ? 1 : 0;
  CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
  return DG_OK;
}
#define DG_LAUNCH(KERNEL, GRID, ...)                          \
  do {                                                        \
    int rc_ = launch_k(c, KERNEL, GRID, bl, __VA_ARGS__);     \
    if (rc_) return rc_;                                      \
  } while (0)

int launch_x2(dg_gpu_ctx* c, cudaEvent_t mid, bool hv = true, bool ht = true) {
  const dim3 bl(c->block), gv(c->blocks_v), gt(c->blocks_t);
  const HalfPair<X2Fn> k = kernels_packed(c->x2, c->kahan, c->x2pm);
  if (!k.v) return fail(DG_ERR_UNSUPPORTED, "no two-shot kernel for this shot count");
  if (hv) DG_LAUNCH(k.v, gv, c->ops2, c->md_f[0], c->d_ctr);
  if (mid) CK(cudaEventRecord(mid, c->stream));
  if (ht) DG_LAUNCH(k.s, gt, c->ops2, c->md_f[0], c->d_ctr);
  return DG_OK;
}

// resident blocks of the persistent wavefront kernel for the current block size
int wave_resident(dg_gpu_ctx* c, int& per_sm) {
  per_sm = 0;
  const WaveFn k = c->wave_async ? kernel_wave_async(c->x2, c->kahan) : kernel_wave(c->x2, c->kahan, true);
  if (!k) return fail(DG_ERR_UNSUPPORTED, "no wavefront step for this shot count");
  if (wave_smem(c) > 48 * 1024) CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wave_smem(c)));
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, c->block, wave_smem(c));
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __LINE__);
  return DG_OK;
}

// shot counts with a wavefront step instance
bool wave_supported(int S) { return S == 2 || S == 4 || S == 8 || S == 16 || S == 32 || S == 64 || S == 128; }

int launch_wave(dg_gpu_ctx* c) {
  const bool as = c->wave_persistent && c->wave_async;
  const WaveFn k = as ? kernel_wave_async(c->x2, c->kahan) : kernel_wave(c->x2, c->kahan, c->wave_persistent);
  if (!k) return fail(DG_ERR_UNSUPPORTED, "no wavefront step for this shot count");
  const dim3 bl(c->block), g(c->wave_persistent ? c->blocks_p : c->blocks_v);
  k<<<g, bl, wave_smem(c), c->stream>>>(c->ops2, c->md_f[0], c->wv, c->d_ctr);
  return DG_OK;
}

// resident blocks of the persistent batch kernel for the current block size
int mx_resident(dg_gpu_ctx* c) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_batch_persistent(c->kahan), c->block, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __LINE__);
  if (per_sm < 1) return fail(DG_ERR_UNSUPPORTED, "the persistent batch kernel does not fit on an SM");
  c->blocks_mxp = per_sm * c->num_sms;
  return DG_OK;
}

// nsteps steps of the FP32 batch in one cooperative launch (all blocks resident, as the grid
// barrier needs)
int launch_mx_p(dg_gpu_ctx* c, int nsteps) {
  MxLoop L{c->d_btab_v, c->d_btab_t, c->blocks_v, c->blocks_t, c->d_mxbar, c->d_mxerr, c->mx_spin, c->mx_extra};
  CK(cudaMemsetAsync(c->d_mxbar, 0, sizeof(unsigned), c->stream));
  const MeshDev<float>* tab = c->d_tab_f;
  void* args[] = {&c->ops_f, &c->ops2, &tab, &L, &c->d_ctr, &nsteps};
  const void* fn = (const void*)kernel_batch_persistent(c->kahan);
  CK(cudaLaunchCooperativeKernel(fn, dim3(c->blocks_mxp), dim3(c->block), args, 0, c->stream));
  return DG_OK;
}

// One step (halves = 3), or only its velocity (1) / stress (2) half for a split mesh.
int launch_step(dg_gpu_ctx* c, cudaEvent_t before_t = nullptr, cudaEvent_t mid = nullptr, cudaEvent_t after = nullptr,
                int halves = 3) {
  const bool hv = halves & 1, ht = halves & 2;
  const dim3 bl(c->block);
  const dim3 gv(c->blocks_v), gt(c->blocks_t);
  cudaStream_t st = c->stream;
  if (before_t) CK(cudaEventRecord(before_t, st));
  // the two launches of a step of family F (mesh table and block table for a batch)
#define DG_TWO(F, OPS, MESH, TAB, BTV, BTT)                                  \
  do {                                                                       \
    if (hv) DG_LAUNCH(F.v, gv, OPS, MESH, TAB, BTV, c->d_ctr);               \
    if (mid) CK(cudaEventRecord(mid, st));                                   \
    if (ht) DG_LAUNCH(F.s, gt, OPS, MESH, TAB, BTT, c->d_ctr);               \
  } while (0)
  if (c->precision == DG_FP64_REF) {
    const HalfPair<GenFn<double>> k = kernels_reference(c->multi, c->ref_otf);
    if (c->multi) DG_TWO(k, c->ops_d, c->md_d[0], c->d_tab_d, c->d_btab_v, c->d_btab_t);
    else DG_TWO(k, c->ops_d, c->md_d[0], (const MeshDev<double>*)nullptr, (const int2*)nullptr, (const int2*)nullptr);
  } else if (c->is_double) {
    const HalfPair<GenFn<double>> k = kernels_fp64(c->multi);
    if (c->multi) DG_TWO(k, c->ops_d, c->md_d[0], c->d_tab_d, c->d_btab_v, c->d_btab_t);
    else DG_TWO(k, c->ops_d, c->md_d[0], (const MeshDev<double>*)nullptr, (const int2*)nullptr, (const int2*)nullptr);
  } else if (c->wave) {  // the whole step in one launch: it is timed as the "velocity" interval
    int rc = launch_wave(c);
    if (rc) return rc;
    if (mid) CK(cudaEventRecord(mid, st));
  } else if (c->mx && c->mx_persistent) {  // the whole step in one launch, timed as the "velocity" interval
    int rc = launch_mx_p(c, 1);
    if (rc) return rc;
    if (mid) CK(cudaEventRecord(mid, st));
  } else if (c->mx) {
    const HalfPair<MxFn> k = kernels_batch(c->kahan);
    if (hv) DG_LAUNCH(k.v, gv, c->ops_f, c->ops2, c->d_tab_f, c->d_btab_v, c->d_ctr);
    if (mid) CK(cudaEventRecord(mid, st));
    if (ht) DG_LAUNCH(k.s, gt, c->ops_f, c->ops2, c->d_tab_f, c->d_btab_t, c->d_ctr);
  } else if (c->x2) {
    int rc = launch_x2(c, mid, hv, ht);
    if (rc) return rc;
  } else {
    const HalfPair<GenFn<float>> k = kernels_fp32(c->kahan, c->multi);
    if (c->multi) DG_TWO(k, c->ops_f, c->md_f[0], c->d_tab_f, c->d_btab_v, c->d_btab_t);
    else DG_TWO(k, c->ops_f, c->md_f[0], (const MeshDev<float>*)nullptr, (const int2*)nullptr, (const int2*)nullptr);
  }
#undef DG_TWO
  CK(cudaGetLastError());
  if (after) CK(cudaEventRecord(after, st));
  return DG_OK;
}

// Capture `steps` steps into an instantiated graph, uploaded now so the first launch does not
// pay for it.
static int capture_steps(dg_gpu_ctx* c, int steps, cudaGraphExec_t* out) {
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = DG_OK;
  for (int k = 0; k < steps && rc == DG_OK; k++) rc = launch_step(c);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __LINE__);
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate", __LINE__);
  CK(cudaGraphUpload(*out, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

int rebuild_graph(dg_gpu_ctx* c) {
  for (cudaGraphExec_t* gp : {&c->graph, &c->graph_small})
    if (*gp) {
      cudaGraphExecDestroy(*gp);
      *gp = nullptr;
    }
  c->graph_small_steps = 0;
  if (c->graph_steps <= 0 || c->mx_persistent) return DG_OK;  // the persistent batch loops on the device
  int rc = capture_steps(c, c->graph_steps, &c->graph);
  if (rc) return rc;
  if (c->graph_steps >= 8) {
    c->graph_small_steps = c->graph_steps / 4;
    if ((rc = capture_steps(c, c->graph_small_steps, &c->graph_small))) return rc;
  }
  c->graph_block = c->block;
  return DG_OK;
}

int set_block(dg_gpu_ctx* c, int block) {
  c->block = block;
  int rc = c->is_double ? layout(c, c->md_d, &c->d_tab_d) : layout(c, c->md_f, &c->d_tab_f);
  if (rc) return rc;
  if (c->wave && (rc = build_wave(c))) {
    if (rc != DG_ERR_UNSUPPORTED) return rc;
    c->wave = false;  // the two-launch step serves this mesh
  }
  if (c->mx && (rc = mx_resident(c))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

// DG_ERR_TIMEOUT if a wavefront wait or a barrier of the persistent batch kernel gave up since
// the last check (then cleared)
int check_wave(dg_gpu_ctx* c) {
  if (c->mx_persistent) {
    int err = 0;
    CK(cudaMemcpyAsync(&err, c->d_mxerr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (err) {
      CK(cudaMemsetAsync(c->d_mxerr, 0, sizeof(int), c->stream));
      return fail(DG_ERR_TIMEOUT, "a grid barrier of the persistent batch step reached its limit");
    }
  }
  if (!c->wave) return DG_OK;
  int err = 0;
  CK(cudaMemcpyAsync(&err, c->wv.error, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (err) {
    CK(cudaMemsetAsync(c->wv.error, 0, sizeof(int), c->stream));
    return fail(DG_ERR_TIMEOUT, "a wait between blocks of the wavefront step reached its limit");
  }
  return DG_OK;
}

int zero_state(dg_gpu_ctx* c) {
  for (size_t k = 0; k < c->mi.size(); k++) {
    const MeshHostInfo& h = c->mi[k];
    const size_t esz = c->is_double ? 8 : 4;
    void* U = c->is_double ? (void*)c->md_d[k].U : (void*)c->md_f[k].U;
    void* C = c->is_double ? (void*)c->md_d[k].C : (void*)c->md_f[k].C;
    void* T = c->is_double ? (void*)c->md_d[k].trace : (void*)c->md_f[k].trace;
    const size_t P = (size_t)h.Kp * h.S_pad;
    CK(cudaMemsetAsync(U, 0, esz * NPLANES * P, c->stream));
    if (C) CK(cudaMemsetAsync(C, 0, esz * NPLANES * P, c->stream));
    CK(cudaMemsetAsync(T, 0, esz * (size_t)h.steps * 2 * std::max(1, h.n_rec) * h.S_pad, c->stream));
  }
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), c->stream));
  if (c->wave) {  // step ids restart at 1: clear the published flags and the tickets
    CK(cudaMemsetAsync(c->wv.vflag, 0, sizeof(unsigned) * (c->wv.NU + 1), c->stream));
    CK(cudaMemsetAsync(c->wv.tickets, 0, sizeof(unsigned long long), c->stream));
    CK(cudaMemsetAsync(c->wv.ptk, 0, sizeof(unsigned) * 2, c->stream));
    CK(cudaMemsetAsync(c->wv.error, 0, sizeof(int), c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->t = 0;
  for (auto& m : c->marks) m.t_end = -1;  // no step mark covers the new run's steps
  return DG_OK;
}

// One schedule the autotuner can pick: threads per block and, for the wavefront step, one block
// per ticket or resident blocks, and the lag margin in warps per SM.
struct TuneChoice {
  int block, persistent, margin;
};

int apply_choice(dg_gpu_ctx* c, const TuneChoice& t) {
  if (c->wave) {
    c->wave_persistent = t.persistent != 0;
    c->margin_warps_per_sm = t.margin;
  }
  if (c->mx) c->mx_persistent = t.persistent != 0;
  int rc = set_block(c, t.block);
  if (rc) return rc;
  return c->mx ? rebuild_graph(c) : DG_OK;
}

// Time each candidate schedule over a few steps from a zero state and keep the fastest; with a
// cache file, reuse (and record) the choice for the same precision, mesh sizes and step form.
// All candidates give the same results bit for bit; only the speed differs.
int autotune(dg_gpu_ctx* c, const char* cache) {
  char key[256];
  long long sumK = 0, sumKS = 0;
  for (auto& h : c->mi) { sumK += h.K; sumKS += (long long)h.K * h.S; }
  snprintf(key, sizeof key, "p%d_m%zu_K%lld_KS%lld_w%d", c->precision, c->mi.size(), sumK, sumKS, c->wave ? 1 : 0);
  if (cache) {
    FILE* f = fopen(cache, "r");
    if (f) {
      char line[512], k2[256];
      TuneChoice t{0, 0, 0};
      while (fgets(line, sizeof line, f))
        if (sscanf(line, "%255s %d %d %d", k2, &t.block, &t.persistent, &t.margin) == 4 && !strcmp(k2, key) &&
            (t.block == 64 || t.block == 128 || t.block == 256) && t.margin > 0 && t.margin <= 64) {
          fclose(f);
          return apply_choice(c, t);
        }
      fclose(f);
    }
  }
  std::vector<TuneChoice> cand;
  for (int b : {64, 128, 256}) {
    if (c->mx) {
      for (int pers = 0; pers < 2; pers++) cand.push_back({b, pers, c->margin_warps_per_sm});
      continue;
    }
    if (!c->wave) {
      cand.push_back({b, 0, c->margin_warps_per_sm});
      continue;
    }
    for (int pers = 0; pers < 2; pers++)
      for (int mw : {8, 10, 14}) cand.push_back({b, pers, mw});
  }
  const long probe = std::min<long>(8, c->max_steps);
  float best = 1e30f;
  TuneChoice best_t = cand[0];
  for (const TuneChoice& t : cand) {
    int rc = apply_choice(c, t);
    if (rc) return rc;
    for (int w = 0; w < 2 && w < probe; w++)
      if ((rc = launch_step(c))) return rc;
    CK(cudaEventRecord(c->ev[0], c->stream));
    for (long k = 2; k < probe; k++)
      if ((rc = launch_step(c))) return rc;
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    if ((rc = check_wave(c))) return rc;
    if (ms < best) { best = ms; best_t = t; }
    if ((rc = zero_state(c))) return rc;
  }
  if (cache) {
    FILE* f = fopen(cache, "a");
    if (f) { fprintf(f, "%s %d %d %d\n", key, best_t.block, best_t.persistent, best_t.margin); fclose(f); }
  }
  return apply_choice(c, best_t);
}

}  // namespace

extern "C" {

void dg_gpu_default_opts(dg_gpu_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->precision = DG_FP64;
  o->device = 0;
  o->reorder = 1;
  o->block_threads = 0;
  o->graph_steps = 0;
  o->autotune = 0;
  o->watchdog_every = 0;
  o->tune_cache = nullptr;
}

const char* dg_gpu_strerror(int code) {
  switch (code) {
    case DG_OK: return "ok";
    case DG_ERR_ARG: return "invalid argument";
    case DG_ERR_CUDA: return "CUDA error";
    case DG_ERR_NOMEM: return "out of memory";
    case DG_ERR_MESH: return "inconsistent mesh arrays";
    case DG_ERR_NONFINITE: return "non-finite values in the wave field";
    case DG_ERR_STATE: return "invalid call for the current state";
    case DG_ERR_UNSUPPORTED: return "unsupported configuration";
    case DG_ERR_NODEVICE: return "no usable sm_100 CUDA device";
    case DG_ERR_ORIENTATION: return "triangle with non-positive Jacobian";
    default: return "unknown error";
  }
}

const char* dg_gpu_last_error(void) { return g_last.c_str(); }

int dg_gpu_init(dg_gpu_ctx** out, const dg_gpu_mesh* meshes, int n_meshes, const dg_gpu_opts* opts_in) {
  if (!out) return fail(DG_ERR_ARG, "ctx pointer is null");
  *out = nullptr;
  if (!meshes || n_meshes < 1) return fail(DG_ERR_ARG, "need at least one mesh");
  if (n_meshes > DG_MAX_MESHES) return fail(DG_ERR_UNSUPPORTED, "too many meshes");
  dg_gpu_opts o;
  if (opts_in) o = *opts_in; else dg_gpu_default_opts(&o);
  if (o.precision < DG_FP64_REF || o.precision > DG_FP32_KAHAN) return fail(DG_ERR_ARG, "unknown precision");
  if (o.block_threads != 0 && o.block_threads != 64 && o.block_threads != 128 && o.block_threads != 256)
    return fail(DG_ERR_ARG, "block_threads must be 0, 64, 128 or 256");

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0)
    return fail(DG_ERR_NODEVICE, "no CUDA device with that ordinal");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, o.device));
  if (prop.major != 10) return fail(DG_ERR_NODEVICE, "the engine is built for sm_100a (B200)");
  CK(cudaSetDevice(o.device));

  std::unique_ptr<dg_gpu_ctx> c(new dg_gpu_ctx());
  c->device = o.device;
  c->num_sms = prop.multiProcessorCount;
  c->precision = o.precision;
  c->is_double = o.precision == DG_FP64_REF || o.precision == DG_FP64;
  c->kahan = o.precision == DG_FP32_KAHAN;
  c->multi = n_meshes > 1;
  c->watchdog_every = std::max(0, o.watchdog_every);
  c->mx = c->multi && !c->is_double;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  // the copy stream (trace fetches, wavelet uploads and snapshots beside the steps) and the
  // step marks exist from the start, so the first fetch pays for neither
  CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  for (auto& m : c->marks) CK(cudaEventCreateWithFlags(&m.ev, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_fetch, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_wavelet, cudaEventDisableTiming));
  for (auto& e : c->ev) CK(cudaEventCreate(&e));

  c->mi.resize(n_meshes);
  double bytes = 0, dof = 0;
  size_t stage = 1, trace_chunk = 0;
  const size_t w = c->is_double ? 8 : 4;
  // the packed FP32 kernels carry the P2 operators as compile-time constants: other operators
  // run on the one-(element, shot)-per-thread kernels
  bool p2_ok = true;
  for (int k = 0; k < n_meshes; k++) p2_ok = p2_ok && p2_operators_match(meshes[k]);
  const int variant = (!c->is_double && !p2_ok && o.variant != 2) ? 1 : o.variant;
  if (o.variant == 2 && !c->is_double && !p2_ok)
    return fail(DG_ERR_UNSUPPORTED, "the packed FP32 kernels need the P2 operators of the reference triangle");
  for (int k = 0; k < n_meshes; k++) {
    Prepared p;
    choose_kind(meshes[k].n_shots, meshes[k].K, !c->is_double, variant, o.wavefront == 1 && n_meshes == 1, p.kind,
                p.S_pad);
    if (o.variant == 2 && p.kind == 0)
      return fail(DG_ERR_UNSUPPORTED, "no packed FP32 kernel for this mesh (FP32 only; at most 128 shots)");
    // the wavefront step: one FP32 mesh on the two-shot kernels; automatic = on
    // automatic: from 16 shots on.  Below, a warp covers several elements and the scattered
    // small gathers in RCM order cost more than the HBM traffic the step saves (200k elements:
    // 2 shots 0.096 ms against 0.073 for two launches, 4 shots 0.103 against 0.091, 8 even,
    // 16 shots 0.199 against 0.228; one shot on 2M elements 0.234 against 0.185)
    c->wave = !c->multi && o.wavefront != -1 &&
              ((p.kind == 2 && wave_supported(p.S_pad) && (p.S_pad >= 16 || o.wavefront == 1)) ||
               (p.kind == 1 && o.wavefront == 1));
    if (o.wavefront == 1 && !c->wave)
      return fail(DG_ERR_UNSUPPORTED, "the wavefront step needs one FP32 mesh with 1, 2, 4, 8, ..., 128 shots");
    const char* arrays = getenv("DG_REF_ARRAYS");
    // rebuilt Dx, Dz for one large one-shot mesh: 200k elements 56.1 against 52.6 G DOF-updates/s,
    // 388k 58.6 against 56.6, and 576 bytes per element less device memory; on 20k elements the
    // register-heavy rebuild is slower (37.3 against 48.8), so small meshes keep the arrays
    const bool want_otf = o.precision == DG_FP64_REF && n_meshes == 1 && meshes[k].n_shots == 1 &&
                          meshes[k].K >= 65536 && !(arrays && atoi(arrays) != 0);
    int rc = prepare(meshes[k], o.precision, c->wave ? 2 : o.reorder, p, want_otf);
    if (n_meshes == 1) c->ref_otf = p.ref_otf;
    if (rc) return rc;
    MeshHostInfo& h = c->mi[k];
    h.K = p.K;
    h.Kp = p.Kp;
    h.S = p.S;
    h.S_pad = p.S_pad;
    h.kind = p.kind;
    if (!c->multi) {
      c->x2 = p.kind == 1 ? 1 : (p.kind >= 2 ? p.S_pad : 0);
      c->x2pm = p.kind == 3;
    }
    if (c->wave) {
      c->face_h = p.face;
      c->rec_elem_h = p.rec_elem;
    }
    h.n_rec = p.n_rec;
    h.steps = meshes[k].n_steps;
    h.dt = meshes[k].dt;
    h.new_of_old = p.new_of_old;
    h.sponge_elems = p.sponge_elems;
    if ((rc = c->upload(&h.d_new_of_old, p.new_of_old))) return rc;
    if (c->is_double) {
      c->md_d.emplace_back();
      if ((rc = upload_mesh<double>(c.get(), meshes[k], p, c->md_d.back()))) return rc;
    } else {
      c->md_f.emplace_back();
      if ((rc = upload_mesh<float>(c.get(), meshes[k], p, c->md_f.back()))) return rc;
    }
    c->max_steps = std::max(c->max_steps, h.steps);
    // algorithmic bytes per step: 90 state values (+60 compensation values) per element and shot
    // (velocity pass reads 30 and writes 12, stress pass reads 30 and writes 18), plus per element
    // geo (2 x 4 values), 1/rho (1 value), lambda/mu/lambda+2mu (4 values) and face codes (2 x 16 B)
    double per = 90.0 * h.S * w + (c->kahan ? 60.0 * h.S * 4 : 0.0) + 13.0 * w + 32.0;
    if (o.precision == DG_FP64_REF) per = 90.0 * h.S * 8 + 2.0 * 72 * 8 + 30 * 8 + 10 * 8 + 32.0;
    // the wavefront step reads and writes each of the 30 values once (the rest is L2 traffic)
    const double per_wave = 60.0 * h.S * w + (c->kahan ? 60.0 * h.S * 4 : 0.0) + 13.0 * w + 32.0;
    bytes += per * (double)h.K;
    c->bytes_wave += per_wave * (double)h.K;
    dof += 30.0 * (double)h.K * h.S;
    stage = std::max(stage, (size_t)std::max<long>(h.K * 6, h.steps * std::max(1, h.n_rec)));
    trace_chunk += (size_t)std::min<long>(100, h.steps) * h.n_rec * h.S;
  }
  // the staging buffer also holds both components of every mesh's traces over 100 steps (one
  // all-mesh fetch per default graph), so fetches of that size need no new allocation
  stage = std::max(stage, 2 * trace_chunk);
  c->bytes_two_pass = bytes;
  c->stats.dof_per_step = dof;
  if (c->is_double) fill_ops(c->ops_d, meshes[0]); else fill_ops(c->ops_f, meshes[0]);
  for (int q = 0; q < 36; q++) {
    c->ops2.Dr[q] = make_float2(c->ops_f.Dr[q], c->ops_f.Dr[q]);
    c->ops2.Ds[q] = make_float2(c->ops_f.Ds[q], c->ops_f.Ds[q]);
  }
  for (int q = 0; q < 54; q++) c->ops2.L[q] = make_float2(c->ops_f.L[q], c->ops_f.L[q]);
  int rc;
  if ((rc = c->alloc(&c->d_ctr, 1))) return rc;
  if ((rc = c->alloc(&c->d_flag, 1))) return rc;
  if ((rc = c->alloc(&c->d_energy, 1))) return rc;
  if ((rc = c->alloc(&c->d_stage, stage))) return rc;
  c->stage_elems = stage;
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), c->stream));

  // automatic block size: 64 threads (measured 2-4 % ahead of 128 and 256 on every family of
  // the time step: small blocks of these latency-bound kernels end and refill SMs sooner), 256
  // for the reference-operator kernels
  // persistent wavefront form on the two-shot layout (200k x 64 batch: FP32 605.5 against 578.5 G
  // DOF-updates/s, FP32-Kahan 370.3 against 364.7, the same bits); the one-shot layout runs
  // slower in it, so that keeps one block per ticket (DG_WAVE_PERSISTENT=0/1 overrides, for tuning)
  c->wave_persistent = c->wave && c->x2 >= 2;
  if (const char* env = getenv("DG_WAVE_PERSISTENT"))
    if (c->wave) c->wave_persistent = atoi(env) != 0;
  // FP32 on the persistent form: the old values staged in shared memory by cp.async (200k x 64
  // batch: 0.6166 against 0.6245 ms a step, the same bits; FP32-Kahan, which stages twice as many,
  // 1.13 against 1.04, keeps the plain form; DG_WAVE_ASYNC=0/1 overrides)
  c->wave_async = c->x2 >= 16 && !c->kahan;
  if (const char* env = getenv("DG_WAVE_ASYNC")) c->wave_async = c->x2 >= 16 && atoi(env) != 0;
  if (const char* env = getenv("DG_PDL")) c->pdl = atoi(env) != 0;
  if (c->mx) {
    if ((rc = c->alloc(&c->d_mxbar, 2))) return rc;
    if ((rc = c->alloc(&c->d_mxerr, 1))) return rc;
    CK(cudaMemsetAsync(c->d_mxbar, 0, 2 * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->d_mxerr, 0, sizeof(int), c->stream));
  }
  // automatic block size: 64 threads for one mesh (see above), 128 for a batch of meshes (its
  // persistent form: 365.5 G DOF-updates/s on the 48-mesh uneven batch against 359.7 at 64
  // threads and 362.8 for two launches a step at 64)
  int block = o.block_threads ? o.block_threads : (o.precision == DG_FP64_REF ? 256 : (c->mx ? 128 : 64));
  if ((rc = set_block(c.get(), block))) return rc;
  // a batch runs persistent when each resident block takes at least 16 work blocks per half, so
  // the two grid barriers of a step cost little against it (DG_MX_PERSISTENT=0/1 overrides)
  if (c->mx) {
    c->mx_persistent = c->blocks_v >= 16LL * c->blocks_mxp;
    if (const char* env = getenv("DG_MX_PERSISTENT")) c->mx_persistent = atoi(env) != 0;
  }
  if (o.autotune && !o.block_threads)
    if ((rc = autotune(c.get(), o.tune_cache))) return rc;
  c->graph_steps = o.graph_steps < 0 ? 0 : (o.graph_steps ? o.graph_steps : (int)std::min<long>(100, c->max_steps));
  if ((rc = rebuild_graph(c.get()))) return rc;
  if ((rc = zero_state(c.get()))) return rc;
  c->stats.block_threads = c->block;
  c->stats.graph_steps = c->graph_steps;
  *out = c.release();
  return DG_OK;
}

// Enqueue n steps on the context stream (graphs where they fit; the watchdog, when on,
// synchronises at its checks).  The caller synchronises.
static int enqueue_steps(dg_gpu_ctx* c, long n, bool timed) {
  c->stats.launches = 0;
  if (timed) { c->stats.ms_velocity = 0; c->stats.ms_stress = 0; }
  long done = 0;
  while (done < n) {
    long chunk = n - done;
    if (c->watchdog_every > 0) {
      long to_check = c->watchdog_every - (c->t % c->watchdog_every);
      chunk = std::min(chunk, to_check);
    }
    if (timed) {
      for (long k = 0; k < chunk; k++) {
        int rc = launch_step(c, c->ev[0], c->ev[1], c->ev[2]);
        if (rc) return rc;
        CK(cudaEventSynchronize(c->ev[2]));
        float a = 0, b = 0;
        CK(cudaEventElapsedTime(&a, c->ev[0], c->ev[1]));
        CK(cudaEventElapsedTime(&b, c->ev[1], c->ev[2]));
        c->stats.ms_velocity += a;
        c->stats.ms_stress += b;
      }
      c->stats.launches += (c->wave || c->mx_persistent ? 1 : 2) * chunk;
    } else if (c->mx_persistent) {
      int rc = launch_mx_p(c, (int)chunk);
      if (rc) return rc;
      c->stats.launches += 1;
    } else {
      long k = 0;
      if (c->graph && c->graph_steps > 0)
        for (; k + c->graph_steps <= chunk; k += c->graph_steps) CK(cudaGraphLaunch(c->graph, c->stream));
      if (c->graph_small && c->graph_small_steps > 0)
        for (; k + c->graph_small_steps <= chunk; k += c->graph_small_steps)
          CK(cudaGraphLaunch(c->graph_small, c->stream));
      for (; k < chunk; k++) {
        int rc = launch_step(c);
        if (rc) return rc;
      }
      c->stats.launches += (c->wave ? 1 : 2) * chunk;
    }
    done += chunk;
    c->t += chunk;
    if (c->watchdog_every > 0 && c->t % c->watchdog_every == 0) {
      CK(cudaMemsetAsync(c->d_flag, 0, sizeof(int), c->stream));
      for (size_t k = 0; k < c->mi.size(); k++) {
        const long long nvals = 30LL * c->mi[k].Kp * c->mi[k].S_pad;
        if (c->is_double) k_nonfinite<double><<<592, 256, 0, c->stream>>>(c->md_d[k].U, nvals, c->d_flag);
        else k_nonfinite<float><<<592, 256, 0, c->stream>>>(c->md_f[k].U, nvals, c->d_flag);
        c->stats.launches++;
      }
      int flag = 0;
      CK(cudaMemcpyAsync(&flag, c->d_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (flag) return fail(DG_ERR_NONFINITE, "NaN or Inf in the velocity fields");
    }
  }
  return DG_OK;
}

static int ensure_copy_stream(dg_gpu_ctx* c) {
  if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  return DG_OK;
}

static int ensure_event(cudaEvent_t* ev) {
  if (!*ev) CK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  return DG_OK;
}

// Records a step mark after the work enqueued so far.
static int mark_steps(dg_gpu_ctx* c) {
  auto& m = c->marks[c->mark_next];
  int rc = ensure_event(&m.ev);
  if (rc) return rc;
  CK(cudaEventRecord(m.ev, c->stream));
  m.t_end = c->t;
  c->mark_next = (c->mark_next + 1) % dg_gpu_ctx::kMarks;
  return DG_OK;
}

// The event after which steps [0, t) are complete: the earliest mark at or past t, else a new
// event after all the work enqueued so far.
static int steps_done_event(dg_gpu_ctx* c, long t, cudaEvent_t* out) {
  const dg_gpu_ctx::StepMark* best = nullptr;
  for (const auto& m : c->marks)
    if (m.ev && m.t_end >= t && m.t_end <= c->t && (!best || m.t_end < best->t_end)) best = &m;
  if (best) {
    *out = best->ev;
    return DG_OK;
  }
  int rc = ensure_event(&c->ev_fetch);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev_fetch, c->stream));
  *out = c->ev_fetch;
  return DG_OK;
}

static int do_steps(dg_gpu_ctx* c, long n, bool timed, bool wait = true) {
  if (!c || n < 0) return fail(DG_ERR_ARG, "bad arguments");
  if (c->half_pending || c->part_done)
    return fail(DG_ERR_STATE, "a half step is waiting for its other half or part");
  if (c->t + n > c->max_steps) return fail(DG_ERR_STATE, "stepping past the end of the wavelet table");
  CK(cudaSetDevice(c->device));
  int rc = enqueue_steps(c, n, timed);
  if (rc) return rc;
  if ((rc = mark_steps(c))) return rc;
  c->stats.steps_done = c->t;
  if (!wait) return DG_OK;
  CK(cudaStreamSynchronize(c->stream));
  return check_wave(c);
}

int dg_gpu_step(dg_gpu_ctx* c, long n) { return do_steps(c, n, false); }
int dg_gpu_step_async(dg_gpu_ctx* c, long n) { return do_steps(c, n, false, false); }
int dg_gpu_synchronize(dg_gpu_ctx* c) {
  if (!c) return fail(DG_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  return check_wave(c);
}
int dg_gpu_step_timed(dg_gpu_ctx* c, long n) { return do_steps(c, n, true); }

static int ensure_flush(dg_gpu_ctx* c) {
  if (c->d_flush) return DG_OK;
  c->flush_bytes = (size_t)256 << 20;  // twice the 126 MB L2
  void* p = nullptr;
  CK(cudaMalloc(&p, c->flush_bytes));
  c->allocs.push_back(p);
  c->d_flush = p;
  return DG_OK;
}

// The staging buffer of at least `elems` doubles.  A larger one is allocated before the smaller
// one is released, so a failed allocation leaves the old buffer in place and the call fails.
static int ensure_stage(dg_gpu_ctx* c, size_t elems) {
  if (c->d_stage && elems <= c->stage_elems) return DG_OK;
  double* p = nullptr;
  int rc = c->alloc(&p, std::max(elems, c->stage_elems));
  if (rc) return rc;
  c->release(c->d_stage);  // the smaller one (after the stream has finished with it)
  c->d_stage = p;
  c->stage_elems = std::max(elems, c->stage_elems);
  return DG_OK;
}

int dg_gpu_step_profiled(dg_gpu_ctx* c, long n, int flush_l2, float* ms_vel, float* ms_str, double* ms_total) {
  if (!c || n < 0) return fail(DG_ERR_ARG, "bad arguments");
  if (c->t + n > c->max_steps) return fail(DG_ERR_STATE, "stepping past the end of the wavelet table");
  CK(cudaSetDevice(c->device));
  int rc;
  if (flush_l2 && (rc = ensure_flush(c))) return rc;
  std::vector<cudaEvent_t> ev((size_t)3 * n);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  for (long k = 0; k < n; k++) {
    if (flush_l2) CK(cudaMemsetAsync(c->d_flush, (int)(k & 0xff), c->flush_bytes, c->stream));
    if ((rc = launch_step(c, ev[3 * k], ev[3 * k + 1], ev[3 * k + 2]))) return rc;
  }
  if (n > 0) CK(cudaEventSynchronize(ev[3 * n - 1]));
  double total = 0, sv = 0, ss = 0;
  for (long k = 0; k < n; k++) {
    float a = 0, b = 0;
    CK(cudaEventElapsedTime(&a, ev[3 * k], ev[3 * k + 1]));
    CK(cudaEventElapsedTime(&b, ev[3 * k + 1], ev[3 * k + 2]));
    if (ms_vel) ms_vel[k] = a;
    if (ms_str) ms_str[k] = b;
    sv += a;
    ss += b;
  }
  if (n > 0 && !flush_l2) {
    float all = 0;
    CK(cudaEventElapsedTime(&all, ev[0], ev[3 * n - 1]));
    total = all;
  } else {
    total = sv + ss;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (ms_total) *ms_total = total;
  c->t += n;
  c->stats.ms_velocity = sv;
  c->stats.ms_stress = ss;
  c->stats.launches = (c->wave ? 1 : 2) * n;
  c->stats.steps_done = c->t;
  return check_wave(c);
}

int dg_gpu_fetch_traces(dg_gpu_ctx* c, int mesh, long t0, long n, double* dst_x, double* dst_z) {
  if (!c || !dst_x || !dst_z || mesh < DG_ALL_MESHES || mesh >= (int)c->mi.size() || t0 < 0 || n < 0)
    return fail(DG_ERR_ARG, "bad arguments");
  // the meshes asked for, their blocks one after the other in both outputs
  const int k0 = mesh == DG_ALL_MESHES ? 0 : mesh, k1 = mesh == DG_ALL_MESHES ? (int)c->mi.size() : mesh + 1;
  long long total = 0;
  for (int k = k0; k < k1; k++) {
    const MeshHostInfo& h = c->mi[k];
    if (t0 + n > std::min(c->t, h.steps)) return fail(DG_ERR_STATE, "trace window beyond the steps taken");
    total += (long long)n * h.n_rec * h.S;
  }
  if (total == 0) return DG_OK;
  CK(cudaSetDevice(c->device));
  int rc = ensure_stage(c, (size_t)2 * total);
  if (rc) return rc;
  // the gather and the copies run on the copy stream after the steps that wrote the window
  // (each step's traces have their own slots), so steps enqueued after those keep running
  cudaEvent_t written = nullptr;
  if ((rc = ensure_copy_stream(c)) || (rc = steps_done_event(c, t0 + n, &written))) return rc;
  cudaStream_t cs = c->copy_stream;
  CK(cudaStreamWaitEvent(cs, written, 0));
  const int B = 256;
  long long at = 0;
  for (int k = k0; k < k1; k++) {
    const MeshHostInfo& h = c->mi[k];
    const long long per = (long long)n * h.n_rec * h.S;
    if (per == 0) continue;
    const int grid = (int)((2 * per + B - 1) / B);
    double* ox = c->d_stage + at;
    double* oz = c->d_stage + total + at;
    if (c->is_double)
      k_fetch_traces<double><<<grid, B, 0, cs>>>(c->md_d[k].trace, h.n_rec, h.S_pad, h.S, t0, n, ox, oz);
    else
      k_fetch_traces<float><<<grid, B, 0, cs>>>(c->md_f[k].trace, h.n_rec, h.S_pad, h.S, t0, n, ox, oz);
    CK(cudaGetLastError());
    at += per;
  }
  CK(cudaMemcpyAsync(dst_x, c->d_stage, total * sizeof(double), cudaMemcpyDeviceToHost, cs));
  CK(cudaMemcpyAsync(dst_z, c->d_stage + total, total * sizeof(double), cudaMemcpyDeviceToHost, cs));
  CK(cudaStreamSynchronize(cs));
  return DG_OK;
}

// Convert Vx and Vz of (mesh, shot) into the reference layout, as doubles, at dst (2 * K * 6).
static int enqueue_velocity_fetch(dg_gpu_ctx* c, int mesh, int shot, double* dst) {
  const MeshHostInfo& h = c->mi[mesh];
  const long long n = h.K * 6;
  const int B = 256, grid = (int)((n + B - 1) / B);
  for (int f = 0; f < 2; f++) {
    if (c->is_double)
      k_fetch_field<double><<<grid, B, 0, c->stream>>>(c->md_d[mesh].U, f * 6, c->md_d[mesh].ES, c->md_d[mesh].PS,
                                                       shot, h.d_new_of_old, (int)h.K, dst + f * n);
    else
      k_fetch_field<float><<<grid, B, 0, c->stream>>>(c->md_f[mesh].U, f * 6, c->md_f[mesh].ES, c->md_f[mesh].PS,
                                                      shot, h.d_new_of_old, (int)h.K, dst + f * n);
  }
  CK(cudaGetLastError());
  return DG_OK;
}

int dg_gpu_step_snapshots(dg_gpu_ctx* c, long n, long every, int mesh, int shot, dg_gpu_snapshot_fn fn,
                          void* user) {
  if (!c || !fn || every <= 0 || n < 0 || n % every || mesh < 0 || mesh >= (int)c->mi.size())
    return fail(DG_ERR_ARG, "bad arguments");
  const MeshHostInfo& h = c->mi[mesh];
  if (shot < 0 || shot >= h.S) return fail(DG_ERR_ARG, "shot out of range");
  if (c->t + n > c->max_steps) return fail(DG_ERR_STATE, "stepping past the end of the wavelet table");
  CK(cudaSetDevice(c->device));
  const size_t per = (size_t)h.K * 6;  // doubles per field
  if (per > c->snap_elems) {            // (re)size the rings: 2 slots x (Vx, Vz)
    if (c->snap_host) {
      CK(cudaFreeHost(c->snap_host));
      c->snap_host = nullptr;
    }
    int rc = c->alloc(&c->snap_dev, 4 * per);
    if (rc) return rc;
    void* hp = nullptr;
    if (cudaMallocHost(&hp, 4 * per * sizeof(double)) != cudaSuccess) return fail(DG_ERR_NOMEM, "pinned snapshot ring");
    c->snap_host = (double*)hp;
    c->snap_elems = per;
  }
  if (int rc = ensure_copy_stream(c)) return rc;
  if (!c->snap_conv[0]) {
    for (int k = 0; k < 2; k++) {
      CK(cudaEventCreateWithFlags(&c->snap_conv[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->snap_copy[k], cudaEventDisableTiming));
    }
  }
  const long J = n / every;
  const long t0 = c->t;
  auto deliver = [&](long j) -> int {
    const int slot = (int)(j & 1);
    CK(cudaEventSynchronize(c->snap_copy[slot]));
    const double* base = c->snap_host + (size_t)slot * 2 * c->snap_elems;
    fn(user, t0 + (j + 1) * every, base, base + per);
    return DG_OK;
  };
  int rc;
  for (long j = 0; j < J; j++) {
    const int slot = (int)(j & 1);
    if ((rc = enqueue_steps(c, every, false))) return rc;
    // the device slot is free once the copy of snapshot j - 2 has finished
    if (j >= 2) CK(cudaStreamWaitEvent(c->stream, c->snap_copy[slot], 0));
    double* dslot = c->snap_dev + (size_t)slot * 2 * c->snap_elems;
    if ((rc = enqueue_velocity_fetch(c, mesh, shot, dslot))) return rc;
    CK(cudaEventRecord(c->snap_conv[slot], c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, c->snap_conv[slot], 0));
    // the host slot is free: the callback of snapshot j - 2 returned before this loop turn
    CK(cudaMemcpyAsync(c->snap_host + (size_t)slot * 2 * c->snap_elems, dslot, 2 * per * sizeof(double),
                       cudaMemcpyDeviceToHost, c->copy_stream));
    CK(cudaEventRecord(c->snap_copy[slot], c->copy_stream));
    // while the device works on snapshot j, hand snapshot j - 1 to the caller
    if (j >= 1 && (rc = deliver(j - 1))) return rc;
  }
  if (J >= 1 && (rc = deliver(J - 1))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->stats.steps_done = c->t;
  return check_wave(c);
}

int dg_gpu_fetch(dg_gpu_ctx* c, int what, int mesh, int shot, double* dst) {
  if (!c || !dst || mesh < 0 || mesh >= (int)c->mi.size()) return fail(DG_ERR_ARG, "bad arguments");
  const MeshHostInfo& h = c->mi[mesh];
  const bool all = shot == DG_ALL_SHOTS && what >= DG_VX && what <= DG_TXZ;
  if (!all && (shot < 0 || shot >= h.S)) return fail(DG_ERR_ARG, "shot out of range");
  CK(cudaSetDevice(c->device));
  const int B = 256;
  if (what >= DG_VX && what <= DG_TXZ) {
    // one shot, or every shot one after the other ([S][K][Np]) with one copy and one wait
    const long long n = h.K * 6;
    const int s0 = all ? 0 : shot, s1 = all ? h.S : shot + 1;
    int rc = ensure_stage(c, (size_t)n * (s1 - s0));
    if (rc) return rc;
    const int grid = (int)((n + B - 1) / B);
    for (int s = s0; s < s1; s++) {
      double* out = c->d_stage + (size_t)(s - s0) * n;
      if (c->is_double)
        k_fetch_field<double><<<grid, B, 0, c->stream>>>(c->md_d[mesh].U, what * 6, c->md_d[mesh].ES, c->md_d[mesh].PS,
                                                         s, h.d_new_of_old, (int)h.K, out);
      else
        k_fetch_field<float><<<grid, B, 0, c->stream>>>(c->md_f[mesh].U, what * 6, c->md_f[mesh].ES, c->md_f[mesh].PS,
                                                        s, h.d_new_of_old, (int)h.K, out);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, c->d_stage, (size_t)n * (s1 - s0) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  } else if (what == DG_TRACE_X || what == DG_TRACE_Z) {
    const long long steps = std::min(c->t, h.steps);
    const long long n = steps * h.n_rec;
    if (n > 0) {
      int rc = ensure_stage(c, (size_t)n);
      if (rc) return rc;
      const int grid = (int)((n + B - 1) / B);
      const int comp = what - DG_TRACE_X;
      if (c->is_double)
        k_fetch_trace<double><<<grid, B, 0, c->stream>>>(c->md_d[mesh].trace, comp, h.n_rec, h.S_pad, shot, steps,
                                                         c->d_stage);
      else
        k_fetch_trace<float><<<grid, B, 0, c->stream>>>(c->md_f[mesh].trace, comp, h.n_rec, h.S_pad, shot, steps,
                                                        c->d_stage);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(dst, c->d_stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
  } else if (what == DG_ENERGY) {
    CK(cudaMemsetAsync(c->d_energy, 0, sizeof(double), c->stream));
    const int grid = (int)((h.K + B - 1) / B);
    if (c->is_double) k_energy<double><<<grid, B, 0, c->stream>>>(c->ops_d, c->md_d[mesh], shot, c->d_energy);
    else k_energy<float><<<grid, B, 0, c->stream>>>(c->ops_f, c->md_f[mesh], shot, c->d_energy);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, c->d_energy, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  } else {
    return fail(DG_ERR_STATE, "unknown fetch item");
  }
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

int dg_gpu_load(dg_gpu_ctx* c, int what, int mesh, int shot, const double* src) {
  if (!c || !src || mesh < 0 || mesh >= (int)c->mi.size()) return fail(DG_ERR_ARG, "bad arguments");
  const MeshHostInfo& h = c->mi[mesh];
  if (shot < 0 || shot >= h.S) return fail(DG_ERR_ARG, "shot out of range");
  if (what < DG_VX || what > DG_TXZ) return fail(DG_ERR_STATE, "only fields can be loaded");
  CK(cudaSetDevice(c->device));
  const long long n = h.K * 6;
  int rc = ensure_stage(c, (size_t)n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->d_stage, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const int B = 256, grid = (int)((n + B - 1) / B);
  if (c->is_double)
    k_load_field<double><<<grid, B, 0, c->stream>>>(c->md_d[mesh].U, c->md_d[mesh].C, what * 6, c->md_d[mesh].ES, c->md_d[mesh].PS,
                                                    shot, h.d_new_of_old, (int)h.K, c->d_stage);
  else
    k_load_field<float><<<grid, B, 0, c->stream>>>(c->md_f[mesh].U, c->md_f[mesh].C, what * 6, c->md_f[mesh].ES, c->md_f[mesh].PS,
                                                   shot, h.d_new_of_old, (int)h.K, c->d_stage);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

int dg_gpu_reset(dg_gpu_ctx* c) {
  if (!c) return fail(DG_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  c->half_pending = false;
  c->part_done = 0;
  return zero_state(c);
}

int dg_gpu_half_step(dg_gpu_ctx* c, int half) {
  if (!c || (half != 0 && half != 1)) return fail(DG_ERR_ARG, "bad arguments");
  if (c->wave) return fail(DG_ERR_UNSUPPORTED, "half steps need the two-launch step (wavefront = -1)");
  if (c->part_done) return fail(DG_ERR_STATE, "the other part of the open half step has not run");
  if ((half == 0) == c->half_pending)
    return fail(DG_ERR_STATE, half == 0 ? "velocity half again before the stress half" : "stress half without the velocity half");
  if (half == 0 && c->t + 1 > c->max_steps) return fail(DG_ERR_STATE, "stepping past the end of the wavelet table");
  CK(cudaSetDevice(c->device));
  int rc = launch_step(c, nullptr, nullptr, nullptr, half == 0 ? 1 : 2);
  if (rc) return rc;
  c->half_pending = half == 0;
  if (half == 1) {
    c->t += 1;
    c->stats.steps_done = c->t;
  }
  return DG_OK;
}

// One part of a half step of mesh 0: the element blocks [0, bB) (boundary) or [bB, bO)
// (interior), bB and bO the first blocks past the lanes of elements part_eB and part_eO.  A
// block holds consecutive lanes of consecutive elements in every one-mesh kernel (lane g of
// element g / lanes-per-element), so each lane of a non-ghost element runs in exactly one part,
// and every element with a ghost neighbour in the boundary part.  The stress part that closes
// the half also runs the recorder blocks.  An empty window launches one block past the element
// blocks (its lanes are out of range and return), so the step counters still advance.
extern "C++" {
template <class R> static void set_window(MeshDev<R>& m, int b0, int b1) {
  m.block0 = b0;
  m.n_elem_blocks = b1;
}
static int launch_part(dg_gpu_ctx* c, int half, int part, bool record) {
  const MeshHostInfo& h = c->mi[0];
  const int B = c->block;
  auto blocks = [&](long n) -> int {
    const long long lanes = h.kind == 1 ? (n + 1) / 2 : (h.kind >= 2 ? n * (long long)(h.S_pad / 2) : n * (long long)h.S_pad);
    return (int)std::min<long long>(h.elem_blocks, (lanes + B - 1) / B);
  };
  const int bB = blocks(c->part_eB), bO = std::max(bB, blocks(c->part_eO));
  int b0 = part == 1 ? 0 : bB, b1 = part == 1 ? bB : bO;
  if (b1 == b0) {
    b0 = h.elem_blocks;
    b1 = h.elem_blocks + 1;
  }
  const int save_v = c->blocks_v, save_t = c->blocks_t;
  c->blocks_v = b1 - b0;
  c->blocks_t = b1 - b0 + (record ? h.rec_blocks : 0);
  if (c->is_double) set_window(c->md_d[0], b0, b1); else set_window(c->md_f[0], b0, b1);
  const int rc = launch_step(c, nullptr, nullptr, nullptr, half == 0 ? 1 : 2);
  c->blocks_v = save_v;
  c->blocks_t = save_t;
  if (c->is_double) set_window(c->md_d[0], 0, h.elem_blocks); else set_window(c->md_f[0], 0, h.elem_blocks);
  return rc;
}
}  // extern "C++"

int dg_gpu_half_step_part(dg_gpu_ctx* c, int half, int part) {
  if (!c || (half != 0 && half != 1) || part < DG_PART_ALL || part > DG_PART_INTERIOR)
    return fail(DG_ERR_ARG, "bad arguments");
  if (part == DG_PART_ALL) return dg_gpu_half_step(c, half);
  if (c->wave) return fail(DG_ERR_UNSUPPORTED, "half steps need the two-launch step (wavefront = -1)");
  if (c->multi) return fail(DG_ERR_UNSUPPORTED, "half-step parts need a context of one mesh");
  if (c->halo.empty()) return fail(DG_ERR_STATE, "no halo lists: the parts are defined by the ghosts");
  if (c->part_done) {
    if (half != c->part_half) return fail(DG_ERR_STATE, "the other part of the open half step has not run");
    if (c->part_done & part) return fail(DG_ERR_STATE, "this part of the half step has already run");
  } else {
    if ((half == 0) == c->half_pending)
      return fail(DG_ERR_STATE, half == 0 ? "velocity half again before the stress half" : "stress half without the velocity half");
    if (half == 0 && c->t + 1 > c->max_steps) return fail(DG_ERR_STATE, "stepping past the end of the wavelet table");
  }
  CK(cudaSetDevice(c->device));
  const bool closes = (c->part_done | part) == 3;
  int rc = launch_part(c, half, part, closes && half == 1);
  if (rc) return rc;
  c->part_done |= part;
  c->part_half = half;
  if (closes) {
    c->part_done = 0;
    c->half_pending = half == 0;
    if (half == 1) {
      c->t += 1;
      c->stats.steps_done = c->t;
    }
  }
  return DG_OK;
}

int dg_gpu_halo_lists(dg_gpu_ctx* c, int mesh, long n_send, const long* send, long n_recv, const long* recv) {
  if (!c || mesh < 0 || mesh >= (int)c->mi.size() || n_send < 0 || n_recv < 0 || (n_send && !send) ||
      (n_recv && !recv))
    return fail(DG_ERR_ARG, "bad arguments");
  const MeshHostInfo& h = c->mi[mesh];
  std::vector<int> a(n_send), b(n_recv);
  for (long k = 0; k < n_send; k++) {
    if (send[k] < 0 || send[k] >= h.K) return fail(DG_ERR_ARG, "send element out of range");
    a[k] = h.new_of_old[send[k]];
  }
  for (long k = 0; k < n_recv; k++) {
    if (recv[k] < 0 || recv[k] >= h.K) return fail(DG_ERR_ARG, "receive element out of range");
    b[k] = h.new_of_old[recv[k]];
  }
  CK(cudaSetDevice(c->device));
  c->halo.resize(c->mi.size());
  dg_gpu_ctx::Halo& hl = c->halo[mesh];
  int rc;
  if (n_send && (rc = c->upload(&hl.d_send, a))) return rc;
  if (n_recv && (rc = c->upload(&hl.d_recv, b))) return rc;
  hl.n_send = n_send;
  hl.n_recv = n_recv;
  if (mesh == 0 && !c->multi) {
    // the parts of a split half step: ghosts are the received elements; the boundary part must
    // hold every element with a ghost face neighbour (it runs after the ghosts are updated)
    std::vector<int4> face(h.Kp);
    const int4* d_face = c->is_double ? c->md_d[0].face : c->md_f[0].face;
    CK(cudaMemcpyAsync(face.data(), d_face, sizeof(int4) * h.Kp, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<char> ghost(h.K, 0);
    for (int x : b) ghost[x] = 1;
    long eB = 0, eO = 0;
    for (long n = 0; n < h.K; n++) {
      if (ghost[n]) continue;
      eO = n + 1;
      const int codes[3] = {face[n].x, face[n].y, face[n].z};
      for (int f = 0; f < 3; f++)
        if (codes[f] >= 0 && ghost[codes[f] >> 4]) eB = n + 1;
    }
    c->part_eB = eB;
    c->part_eO = eO;
  }
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

// what 0: the velocity planes (Vx, Vz: 12), 1: the stress planes (Txx, Tzz, Txz: 18)
static int halo_copy(dg_gpu_ctx* c, int mesh, int what, void* buf, bool pack, bool sync = true) {
  if (!c || mesh < 0 || mesh >= (int)c->mi.size() || (what != 0 && what != 1))
    return fail(DG_ERR_ARG, "bad arguments");
  if ((int)c->halo.size() <= mesh) return fail(DG_ERR_STATE, "no halo lists for this mesh");
  const dg_gpu_ctx::Halo& hl = c->halo[mesh];
  const long n = pack ? hl.n_send : hl.n_recv;
  if (n == 0) return DG_OK;
  if (!buf) return fail(DG_ERR_ARG, "null buffer");
  const MeshHostInfo& h = c->mi[mesh];
  const int plane0 = what == 0 ? 0 : 12, planes = what == 0 ? 12 : 18;
  const long long total = (long long)n * planes * h.S;
  const int B = 256;
  const unsigned grid = (unsigned)((total + B - 1) / B);
  CK(cudaSetDevice(c->device));
  const int* el = pack ? hl.d_send : hl.d_recv;
  if (c->is_double) {
    const MeshDev<double>& m = c->md_d[mesh];
    if (pack) k_halo_pack<double><<<grid, B, 0, c->stream>>>(m.U, m.ES, m.PS, h.S, plane0, planes, el, (int)n, (double*)buf);
    else k_halo_unpack<double><<<grid, B, 0, c->stream>>>(m.U, m.ES, m.PS, h.S, plane0, planes, el, (int)n, (const double*)buf);
  } else {
    const MeshDev<float>& m = c->md_f[mesh];
    if (pack) k_halo_pack<float><<<grid, B, 0, c->stream>>>(m.U, m.ES, m.PS, h.S, plane0, planes, el, (int)n, (float*)buf);
    else k_halo_unpack<float><<<grid, B, 0, c->stream>>>(m.U, m.ES, m.PS, h.S, plane0, planes, el, (int)n, (const float*)buf);
  }
  CK(cudaGetLastError());
  if (pack && sync) CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

int dg_gpu_halo_pack(dg_gpu_ctx* c, int mesh, int what, void* buf) { return halo_copy(c, mesh, what, buf, true); }
int dg_gpu_halo_pack_async(dg_gpu_ctx* c, int mesh, int what, void* buf) {
  return halo_copy(c, mesh, what, buf, true, false);
}
void* dg_gpu_context_stream(dg_gpu_ctx* c) { return c ? (void*)c->stream : nullptr; }
int dg_gpu_halo_unpack(dg_gpu_ctx* c, int mesh, int what, const void* buf) {
  return halo_copy(c, mesh, what, const_cast<void*>(buf), false);
}

int dg_gpu_debug_stall_wave(dg_gpu_ctx* c, int unit) {
  if (!c) return fail(DG_ERR_ARG, "null context");
  if (c->mx_persistent) {  // the grid barrier waits for one arrival more than the grid holds
    c->mx_extra = unit >= 0 ? 1u : 0u;
    c->mx_spin = unit >= 0 ? (1u << 14) : (1u << 22);
    return DG_OK;
  }
  if (!c->wave) return fail(DG_ERR_UNSUPPORTED, "this context has no wavefront step");
  if (unit >= c->wv.NU) return fail(DG_ERR_ARG, "unit out of range");
  CK(cudaSetDevice(c->device));
  int* slot = const_cast<int*>(c->wv.wait);
  if (c->stall_unit >= 0) {  // put the replaced entry back
    CK(cudaMemcpyAsync(slot + (size_t)c->stall_unit * c->wv.W, &c->stall_saved, sizeof(int),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->stall_unit = -1;
  }
  if (unit >= 0) {
    const int never = c->wv.NU;
    CK(cudaMemcpyAsync(&c->stall_saved, slot + (size_t)unit * c->wv.W, sizeof(int), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaMemcpyAsync(slot + (size_t)unit * c->wv.W, &never, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->stall_unit = unit;
  }
  return DG_OK;
}

int dg_gpu_set_wavelet(dg_gpu_ctx* c, int mesh, long t0, long n, const double* w) {
  if (!c || !w || mesh < DG_ALL_MESHES || mesh >= (int)c->mi.size() || t0 < 0 || n < 0)
    return fail(DG_ERR_ARG, "bad arguments");
  const int k0 = mesh == DG_ALL_MESHES ? 0 : mesh, k1 = mesh == DG_ALL_MESHES ? (int)c->mi.size() : mesh + 1;
  for (int k = k0; k < k1; k++)
    if (t0 + n > c->mi[k].steps) return fail(DG_ERR_ARG, "wavelet window beyond a mesh's steps");
  CK(cudaSetDevice(c->device));
  // samples that no enqueued step reads (t0 at or past the steps enqueued so far) go over the
  // copy stream, and the context stream waits for them, so steps in flight keep running;
  // otherwise the copy follows the enqueued steps on the context stream
  const bool ahead = t0 >= c->t;
  int rc;
  if (ahead && ((rc = ensure_copy_stream(c)) || (rc = ensure_event(&c->ev_wavelet)))) return rc;
  cudaStream_t st = ahead ? c->copy_stream : c->stream;
  for (int k = k0; k < k1; k++) {  // mesh k's samples follow those of the meshes before it
    const double* dw = c->is_double ? c->md_d[k].wavelet : c->md_f[k].wavelet;
    CK(cudaMemcpyAsync((void*)(dw + t0), w + (size_t)(k - k0) * n, n * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  if (ahead) {
    CK(cudaEventRecord(c->ev_wavelet, st));
    CK(cudaStreamWaitEvent(c->stream, c->ev_wavelet, 0));
  }
  CK(cudaStreamSynchronize(st));
  return DG_OK;
}

int dg_gpu_flush_l2(dg_gpu_ctx* c) {
  if (!c) return fail(DG_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  int rc = ensure_flush(c);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->d_flush, (int)(c->t & 0xff), c->flush_bytes, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DG_OK;
}

int dg_gpu_stats_get(dg_gpu_ctx* c, dg_gpu_stats* out) {
  if (!c || !out) return fail(DG_ERR_ARG, "bad arguments");
  c->stats.steps_done = c->t;
  c->stats.block_threads = c->block;
  c->stats.graph_steps = c->graph_steps;
  c->stats.kernel_family =
      c->precision == DG_FP64_REF
          ? 0
          : (c->wave ? (c->wave_persistent ? 6 : 5)
                     : (c->mx ? (c->mx_persistent ? 8 : 4) : (c->x2 == 1 ? 3 : (c->x2 ? (c->x2pm ? 7 : 2) : 1))));
  c->stats.bytes_per_step = c->wave ? c->bytes_wave : c->bytes_two_pass;
  *out = c->stats;
  return DG_OK;
}

long dg_gpu_steps_done(dg_gpu_ctx* c) { return c ? c->t : -1; }

int dg_gpu_free(dg_gpu_ctx* c) {
  if (!c) return DG_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete c;
  return DG_OK;
}

}  // extern "C"
