// Allocation-free variant of the CFL_MAX local time step.
//
// Some callers of this library cannot call cudaMalloc: solvers embedded in a
// host application that owns all device memory through its own pool, code
// running inside a captured or externally scheduled stream where allocation
// calls are not allowed, and drivers that preallocate everything at start-up
// and forbid later allocations.  fcfd_local_dt (fcfd.cu) needs scratch memory
// for the global minimum of the CFL_MAX mode, which it takes from the context's
// cudaMalloc'd buffers; this entry point keeps that scratch in a file-scope
// __device__ array instead, so it allocates nothing.
//
// Scratch: g_dt_scratch holds one partial minimum per block of the first pass
// plus one slot for the global minimum.  It is a fixed size (kMaxBlocks + 32
// doubles, 33 KB), so at most kMaxBlocks * kThreads cells are accepted.  Every
// GPU that loads the library holds the array until the process exits.  Every
// slot a call reads is written earlier in the same call, so nothing needs
// clearing, but all calls share the one array: calls that overlap on the GPU
// (different streams, or different host threads) race on it and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "internal.hpp"

namespace fcfd {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;
constexpr int64_t kMaxCells = (int64_t)kMaxBlocks * kThreads;  // 1,048,576 cells
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dt_scratch[kMaxBlocks + 32];

// Host-side copy of each device's scratch address, resolved once per device.
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

struct Gas {
  double gamma, R, Pref, Tref, cfl;
};

// dt_c = cfl * l_c / (|V| + a) (time_step.cc:181-186) and per-block minima.
__global__ void k_dt_cells(const double *__restrict__ W, const double *__restrict__ len, int nc, Gas g,
                           double *__restrict__ dt, double *__restrict__ scratch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double v = INFINITY;
  if (c < nc) {
    const double p = W[5 * c], u = W[5 * c + 1], vv = W[5 * c + 2], w = W[5 * c + 3], T = W[5 * c + 4];
    const double rho = (p + g.Pref) / (g.R * (T + g.Tref));
    const double a = sqrt(g.gamma * (p + g.Pref) / rho);
    v = g.cfl * len[c] / (sqrt(u * u + vv * vv + w * w) + a);
    dt[c] = v;
  }
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double sh[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sh[0];
    for (int k = 1; k < kThreads / 32; ++k) m = fmin(m, sh[k]);
    scratch[blockIdx.x] = m;
  }
}

// One block reduces the partial minima into scratch[kMaxBlocks].
__global__ void k_dt_reduce(int nblocks, double *__restrict__ scratch) {
  double v = INFINITY;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) v = fmin(v, scratch[i]);
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double sh[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sh[0];
    for (int k = 1; k < kThreads / 32; ++k) m = fmin(m, sh[k]);
    scratch[kMaxBlocks] = m;
  }
}

__global__ void k_dt_fill(int nc, double *__restrict__ dt, const double *__restrict__ scratch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) dt[c] = scratch[kMaxBlocks];
}

// Device address of g_dt_scratch for the current device (first call on a
// device resolves it with cudaGetSymbolAddress).
double *scratch_for_current_device(std::string &err) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return nullptr; }
  if (dev < 0 || dev >= kMaxDevices) { err = "device index out of range"; return nullptr; }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    double *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_dt_scratch);
    if (e != cudaSuccess || !ptr) {
      err = std::string("cudaGetSymbolAddress(g_dt_scratch): ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_scratch_addr[dev] = ptr;
  }
  return g_scratch_addr[dev];
}

}  // namespace
}  // namespace fcfd

extern "C" int fcfd_local_dt_cflmax_noalloc(const double *W, const double *length, int32_t n_cells, double gamma,
                                            double gas_R, double Pref, double Tref, double cfl, double *dt,
                                            void *stream) {
  using namespace fcfd;
  if (n_cells < 0 || !W || !length || !dt) {
    set_last_error("fcfd_local_dt_cflmax_noalloc: null pointer or negative cell count");
    return FCFD_ERR_INPUT;
  }
  if ((int64_t)n_cells > kMaxCells) {
    set_last_error("fcfd_local_dt_cflmax_noalloc: " + std::to_string(n_cells) + " cells exceed the static scratch limit of " +
                   std::to_string(kMaxCells) + " cells");
    return FCFD_ERR_INPUT;
  }
  if (n_cells == 0) return FCFD_OK;
  std::string err;
  double *scratch = scratch_for_current_device(err);
  if (!scratch) {
    set_last_error(err);
    return FCFD_ERR_CUDA;
  }
  // An error left by the caller's earlier work is reported as such and left
  // in place for the caller's own check; only errors of the launches below
  // are taken (and cleared) here.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    set_last_error(std::string("fcfd_local_dt_cflmax_noalloc: a CUDA error from earlier work on this thread is "
                               "pending (nothing launched): ") + cudaGetErrorString(e));
    return FCFD_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nblocks = (n_cells + kThreads - 1) / kThreads;
  const Gas g{gamma, gas_R, Pref, Tref, cfl};
  k_dt_cells<<<nblocks, kThreads, 0, s>>>(W, length, n_cells, g, dt, scratch);
  k_dt_reduce<<<1, kThreads, 0, s>>>(nblocks, scratch);
  k_dt_fill<<<nblocks, kThreads, 0, s>>>(n_cells, dt, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(std::string("fcfd_local_dt_cflmax_noalloc: launch failed: ") + cudaGetErrorString(e));
    return FCFD_ERR_CUDA;
  }
  return FCFD_OK;
}
