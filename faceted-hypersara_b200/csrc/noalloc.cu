// Allocation-free l2-ball projection (device pointers, static scratch).
//
// Callers that must not allocate device memory use this entry point: host
// frameworks that own the whole device heap through their own pool (MATLAB
// gpuArray, PyTorch's caching allocator) and real-time pipelines that forbid
// allocation after start-up.  The caller
// passes device buffers for the inputs and the output; the partial sums of
// ||x - y||^2 live in a file-scope device array that every call on a device
// shares.
#include <cmath>
#include <mutex>
#include <algorithm>

#include "common.cuh"

namespace fhs {

namespace {

constexpr int kChunk = 4096;                    // doubles reduced per partial sum
constexpr int64_t kScratch = 65536;             // 512 KB of scratch per device
constexpr int64_t kMaxPartials = kScratch - 1;  // last slot holds the scale
constexpr int64_t kMaxComplex = kMaxPartials * kChunk / 2;

// Slots [0, nparts) hold the partial sums of one call and slot kScratch-1 its
// scale factor; every slot a call reads is written by the same call first, so
// nothing needs clearing between calls.
static __device__ __align__(256) double g_l2ball_partials[kScratch];

std::mutex g_setup_mutex;
double* g_partials_addr[64] = {nullptr};

__global__ void __launch_bounds__(256) chunk_sumsq_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                          int64_t m, double* __restrict__ partials) {
  __shared__ double sh[256];
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  double a = 0.0;
  for (int k = threadIdx.x; k < kChunk; k += blockDim.x) {
    const int64_t i = base + k;
    if (i < m) {
      const double d = x[i] - y[i];
      a += d * d;
    }
  }
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(256) scale_kernel(double* __restrict__ partials, int nparts, double eps) {
  __shared__ double sh[256];
  double a = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) a += partials[k];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double nrm = sqrt(sh[0]);
    partials[kScratch - 1] = nrm > 0 ? fmin(eps / nrm, 1.0) : 1.0;
  }
}

__global__ void __launch_bounds__(256) project_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                      int64_t m, const double* __restrict__ partials,
                                                      double* __restrict__ p) {
  const double scale = partials[kScratch - 1];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = y[i] + (x[i] - y[i]) * scale;
}

// Set-up, once per device with that device current: the device address of
// the scratch array (the host-side symbol is only a stand-in for it), and
// the three kernels' module loaded now (cudaFuncGetAttributes), so that no
// later call loads code on the GPU -- with lazy module loading a kernel is
// otherwise loaded at its first launch, which could fall inside a stream
// capture.  The address is cached for the life of the process and belongs
// to the device's primary context: after cudaDeviceReset() on that device it
// is stale, and calls are not supported.
double* scratch_address(int device) {
  FHS_CHECK(device >= 0 && device < 64, FHS_ERR_UNSUPPORTED, "device index >= 64");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_l2ball_partials);
    if (e != cudaSuccess)
      throw Error(FHS_ERR_CUDA, std::string("cudaGetSymbolAddress(l2-ball scratch): ") + cudaGetErrorString(e));
    cudaFuncAttributes fa;
    FHS_CUDA(cudaFuncGetAttributes(&fa, chunk_sumsq_kernel));
    FHS_CUDA(cudaFuncGetAttributes(&fa, scale_kernel));
    FHS_CUDA(cudaFuncGetAttributes(&fa, project_kernel));
    g_partials_addr[device] = static_cast<double*>(p);
  }
  return g_partials_addr[device];
}

}  // namespace

}  // namespace fhs

using namespace fhs;

extern "C" fhs_status fhs_proj_l2ball_noalloc(int device, int64_t n, const double* x, double eps, const double* y,
                                              double* p, void* stream) {
  try {
    FHS_CHECK(n >= 0, FHS_ERR_INVALID_ARG, "n must be >= 0");
    FHS_CHECK(n <= kMaxComplex, FHS_ERR_UNSUPPORTED,
              "fhs_proj_l2ball_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                  std::to_string(kMaxComplex) + " complex entries; use fhs_proj_l2ball");
    FHS_CHECK(x && y && p, FHS_ERR_INVALID_ARG, "null device pointer");
    FHS_CHECK(std::isfinite(eps) && eps >= 0, FHS_ERR_INVALID_ARG, "eps must be finite and >= 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(FHS_ERR_NO_DEVICE, "no CUDA device");
    FHS_CHECK(device >= 0 && device < ndev, FHS_ERR_INVALID_ARG, "bad device index");
    DeviceGuard g(device);
    double* partials = scratch_address(device);
    if (n == 0) {
      set_last_error("");
      return FHS_OK;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t m = 2 * n;  // interleaved (re, im)
    const int nparts = (int)((m + kChunk - 1) / kChunk);
    chunk_sumsq_kernel<<<nparts, 256, 0, s>>>(x, y, m, partials);
    count_launch();
    FHS_LAUNCH_CHECK();
    scale_kernel<<<1, 256, 0, s>>>(partials, nparts, eps);
    count_launch();
    FHS_LAUNCH_CHECK();
    const int blocks = (int)std::min<int64_t>((m + 255) / 256, 148 * 8);
    project_kernel<<<blocks, 256, 0, s>>>(x, y, m, partials, p);
    count_launch();
    FHS_LAUNCH_CHECK();
    set_last_error("");
    return FHS_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FHS_ERR_INVALID_ARG;
  }
}
