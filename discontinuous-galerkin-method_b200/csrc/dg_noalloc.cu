// dg_noalloc.cu — wavefield energy for callers that cannot allocate device memory.
//
// dg_gpu_energy_noalloc computes the same FP64 energy as dg_gpu_fetch(DG_ENERGY) from fields the
// caller already holds in device memory, and keeps its partial sums in a file-scope static
// device array instead of a cudaMalloc'd buffer.  Host code must not use g_partials' name as a
// device address: it is a host-side stand-in.  The device address is looked up with
// cudaGetSymbolAddress, with the device current, on the first call on each device and again
// whenever that device's current context is no longer the one the address was taken in (after
// a cudaDeviceReset by the host program), and handed to the kernels.
#include "dg_gpu.h"

#include <cuda.h>  // CUcontext and CUresult only: the driver call is found at run time
#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace dg {
void set_last_error(const char* msg);  // dg_gpu.cu: the text dg_gpu_last_error() returns
}

namespace {

constexpr int kBlock = 256;
constexpr long kMaxPartials = DG_NOALLOC_MAX_ELEMENTS / kBlock;  // 16384 doubles = 128 KiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxPartials];

std::mutex g_mu;
struct Slot {
  void* ctx = nullptr;     // the context the address was taken in
  double* addr = nullptr;  // g_partials' device address there
};
Slot g_slot[kMaxDevices];

struct Mass {
  double M[36];  // reference mass matrix inv(V V^T) = inverV^T inverV
};

// One partial sum per block: 1/2 J sum_ij M_ij [rho v_i.v_j + compliance(sigma_i, sigma_j)].
__global__ void k_energy_partials(const __grid_constant__ Mass mass, long K, const double* __restrict__ Vx,
                                  const double* __restrict__ Vz, const double* __restrict__ Txx,
                                  const double* __restrict__ Tzz, const double* __restrict__ Txz,
                                  const double* __restrict__ Jacobi, const double* __restrict__ A,
                                  double* __restrict__ partials) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double local = 0.0;
  if (e < K) {
    const double J = Jacobi[e];
    const double rho = 1.0 / A[e * 5 + 0], lam = A[e * 5 + 3], mu = A[e * 5 + 4];
    const double det = 4.0 * mu * (lam + mu);
    double f[5][6];
    const double* src[5] = {Vx, Vz, Txx, Tzz, Txz};
#pragma unroll
    for (int c = 0; c < 5; c++)
#pragma unroll
      for (int i = 0; i < 6; i++) f[c][i] = src[c][e * 6 + i];
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
      for (int k = 0; k < 6; k++) {
        double w = rho * (f[0][i] * f[0][k] + f[1][i] * f[1][k]);
        if (mu > 0.0) {
          w += ((lam + 2 * mu) * (f[2][i] * f[2][k] + f[3][i] * f[3][k]) -
                lam * (f[2][i] * f[3][k] + f[3][i] * f[2][k])) / det +
               f[4][i] * f[4][k] / mu;
        } else if (lam > 0.0) {
          w += (f[2][i] + f[3][i]) * (f[2][k] + f[3][k]) / (4.0 * lam);
        }
        local += 0.5 * J * mass.M[i * 6 + k] * w;
      }
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  __shared__ double red[kBlock / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kBlock / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;  // every block writes its slot
  }
}

// Sum of the n partials in a fixed order (one block), so equal inputs give equal bits.
__global__ void k_energy_finish(const double* __restrict__ partials, int n, double* __restrict__ out) {
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) v += partials[q];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < (int)(blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) *out = w;
  }
}

int fail(int code, const char* msg) {
  dg::set_last_error(msg);
  return code;
}

int cuda_fail(const char* what, cudaError_t e) {
  dg::set_last_error((std::string(what) + ": " + cudaGetErrorString(e)).c_str());
  return DG_ERR_CUDA;
}

// The current driver context as an opaque key, or null where the driver entry point is not
// available (then the address is taken once per device and kept).
void* current_context() {
  using GetCurrent = CUresult (*)(CUcontext*);
  static GetCurrent fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (GetCurrent) nullptr;
    return reinterpret_cast<GetCurrent>(p);
  }();
  CUcontext ctx = nullptr;
  if (!fn || fn(&ctx) != CUDA_SUCCESS) return nullptr;
  return ctx;
}

// Device address of g_partials on `device`, which the caller has made current.  Taken on the
// first call on the device and again when the device's context has changed since.
int scratch_on(int device, double** addr) {
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_mu);
  Slot& sl = g_slot[device];
  if (!sl.addr || sl.ctx != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress", e);
    if (!p) return fail(DG_ERR_CUDA, "cudaGetSymbolAddress gave no address");
    sl.addr = static_cast<double*>(p);
    sl.ctx = ctx;
  }
  *addr = sl.addr;
  return DG_OK;
}

// Makes `device` current for the life of the object and puts the caller's device back after.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) err = cudaSetDevice(device);
  }
  ~DeviceScope() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
};

int energy_on_device(int device, long K, const double* Vx, const double* Vz, const double* Txx,
                     const double* Tzz, const double* Txz, const double* Jacobi, const double* A,
                     const double* inverV, double* out, void* stream) {
  double* partials = nullptr;
  int rc = scratch_on(device, &partials);
  if (rc) return rc;
  Mass mass;
  for (int i = 0; i < 6; i++)
    for (int k = 0; k < 6; k++) {
      double a = 0;
      for (int q = 0; q < 6; q++) a += inverV[q * 6 + i] * inverV[q * 6 + k];
      mass.M[i * 6 + k] = a;
    }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int blocks = (int)((K + kBlock - 1) / kBlock);
  // launched through cudaLaunchKernel so each launch's own status is checked and an error the
  // host program left pending in the runtime is neither returned nor cleared here
  void* a1[] = {&mass, &K, &Vx, &Vz, &Txx, &Tzz, &Txz, &Jacobi, &A, &partials};
  cudaError_t e = cudaLaunchKernel((const void*)k_energy_partials, dim3(blocks), dim3(kBlock), a1, 0, st);
  if (e != cudaSuccess) return cuda_fail("dg_gpu_energy_noalloc: partial sums", e);
  void* a2[] = {&partials, &blocks, &out};
  e = cudaLaunchKernel((const void*)k_energy_finish, dim3(1), dim3(1024), a2, 0, st);
  if (e != cudaSuccess) return cuda_fail("dg_gpu_energy_noalloc: final sum", e);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail("dg_gpu_energy_noalloc", e);
  return DG_OK;
}

}  // namespace

extern "C" int dg_gpu_energy_noalloc(int device, long K, const double* Vx, const double* Vz, const double* Txx,
                                     const double* Tzz, const double* Txz, const double* Jacobi, const double* A,
                                     const double* inverV, double* out, void* stream) {
  if (device < 0 || device >= kMaxDevices) return fail(DG_ERR_ARG, "device ordinal out of range");
  if (K <= 0) return fail(DG_ERR_ARG, "K must be positive");
  if (K > DG_NOALLOC_MAX_ELEMENTS)
    return fail(DG_ERR_ARG, "K exceeds DG_NOALLOC_MAX_ELEMENTS (4,194,304): the static scratch is too small");
  if (!Vx || !Vz || !Txx || !Tzz || !Txz || !Jacobi || !A || !inverV || !out)
    return fail(DG_ERR_ARG, "null pointer");
  DeviceScope scope(device);
  if (scope.err != cudaSuccess) return fail(DG_ERR_NODEVICE, "cannot make the device current");
  return energy_on_device(device, K, Vx, Vz, Txx, Tzz, Txz, Jacobi, A, inverV, out, stream);
}
