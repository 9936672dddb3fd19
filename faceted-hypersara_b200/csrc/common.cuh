// Shared definitions for the B200 Faceted HyperSARA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <stdexcept>

#include "../../include/fhs_b200.h"

namespace fhs {

// Error carried through the C-ABI: every entry point catches it and turns it
// into an fhs_status plus a thread-local message.
struct Error : public std::runtime_error {
  fhs_status status;
  Error(fhs_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);

#define FHS_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      throw ::fhs::Error(FHS_ERR_CUDA, std::string(#call) + ": " +              \
                                           cudaGetErrorString(e_));             \
  } while (0)

#define FHS_CUFFT(call)                                                         \
  do {                                                                          \
    cufftResult r_ = (call);                                                    \
    if (r_ != CUFFT_SUCCESS)                                                    \
      throw ::fhs::Error(FHS_ERR_CUDA, std::string(#call) + ": cufft error " +  \
                                           std::to_string((int)r_));            \
  } while (0)

#define FHS_CHECK(cond, status, msg)                                            \
  do {                                                                          \
    if (!(cond)) throw ::fhs::Error(status, msg);                               \
  } while (0)

// Device buffer owned by a handle (RAII, no implicit copies).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) return;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      throw Error(FHS_ERR_OUT_OF_MEMORY,
                  "cudaMalloc(" + std::to_string(count * sizeof(T)) + " B): " + cudaGetErrorString(e));
    }
    n = count;
  }
  void zero(cudaStream_t s) {
    if (p) FHS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    FHS_CHECK(count <= n, FHS_ERR_INVALID_ARG, "upload larger than buffer");
    if (count) FHS_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t count, cudaStream_t s) const {
    FHS_CHECK(count <= n, FHS_ERR_INVALID_ARG, "download larger than buffer");
    if (count) FHS_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void download_at(T* h, size_t first, size_t count, cudaStream_t s) const {
    FHS_CHECK(first + count <= n, FHS_ERR_INVALID_ARG, "download beyond buffer");
    if (count) FHS_CUDA(cudaMemcpyAsync(h, p + first, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
};

// Makes a device current for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (dev != prev) FHS_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Kernel launch counter (the bench reports how many library kernels ran).
extern unsigned long long g_launches;
inline void count_launch(unsigned n = 1) { g_launches += n; }

#define FHS_LAUNCH_CHECK() FHS_CUDA(cudaGetLastError())

constexpr int kTableSamples = 1024;   // min-max coefficient table samples per grid unit
constexpr int kMaxTaps = 8;           // J <= 8 (the operator uses 7)
constexpr int kBinCells = 8;          // visibility sub-bin edge (grid cells)
constexpr int kTileCells = 64;        // gridding / degridding tile edge (grid cells)
constexpr int kSubPerTile = kTileCells / kBinCells;
constexpr int kMaxBlocksPerChannel = 16;

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace fhs
