// Conversion kernels between the host (MATLAB) formats and the device layout.
#include "apikern.cuh"

#include <algorithm>

namespace fhs {

namespace {

int nblk(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

__global__ void d2f_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void f2d_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

__global__ void vis_gather_kernel(const double* __restrict__ in, float2* __restrict__ out,
                                  const int32_t* __restrict__ perm, const int64_t* __restrict__ ch_voff,
                                  const int32_t* __restrict__ ch_M, int c0, int64_t host_off0) {
  const int ch = c0 + blockIdx.y;
  const int64_t vo = ch_voff[ch];
  const int M = ch_M[ch];
  const int64_t ho = vo - ch_voff[c0] + host_off0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t src = ho + perm[vo + i];
    out[vo + i] = make_float2((float)in[2 * src], (float)in[2 * src + 1]);
  }
}

__global__ void vis_scatter_kernel(const float2* __restrict__ in, double* __restrict__ out,
                                   const int32_t* __restrict__ perm, const int64_t* __restrict__ ch_voff,
                                   const int32_t* __restrict__ ch_M, int c0, int64_t host_off0) {
  const int ch = c0 + blockIdx.y;
  const int64_t vo = ch_voff[ch];
  const int M = ch_M[ch];
  const int64_t ho = vo - ch_voff[c0] + host_off0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dst = ho + perm[vo + i];
    const float2 v = in[vo + i];
    out[2 * dst] = v.x;
    out[2 * dst + 1] = v.y;
  }
}

__device__ __forceinline__ void rho(int ky, int kx, int Ny, int Nx, int Ky, int Kx, double* c, double* s) {
  const long long ay = ((long long)ky * Ny) % (2LL * Ky);
  const long long ax = ((long long)kx * Nx) % (2LL * Kx);
  const double a = (double)ay / Ky + (double)ax / Kx;
  sincospi(a, s, c);
}

__global__ void grid_from_matlab_kernel(const double* __restrict__ in, float2* __restrict__ out, int Ny, int Nx,
                                        int Ky, int Kx) {
  const int64_t No = (int64_t)Ky * Kx;
  const int p = blockIdx.y;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < No; k += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(k / Ky), ky = (int)(k - (int64_t)kx * Ky);
    double c, s;
    rho(ky, kx, Ny, Nx, Ky, Kx, &c, &s);
    const double re = in[2 * (p * No + k)], im = in[2 * (p * No + k) + 1];
    out[p * No + k] = make_float2((float)(c * re - s * im), (float)(c * im + s * re));
  }
}

__global__ void grid_to_matlab_kernel(const float2* __restrict__ in, double* __restrict__ out, int Ny, int Nx,
                                      int Ky, int Kx) {
  const int64_t No = (int64_t)Ky * Kx;
  const int p = blockIdx.y;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < No; k += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(k / Ky), ky = (int)(k - (int64_t)kx * Ky);
    double c, s;
    rho(ky, kx, Ny, Nx, Ky, Kx, &c, &s);
    const float2 v = in[p * No + k];
    // conj(rho) * v
    out[2 * (p * No + k)] = c * v.x + s * v.y;
    out[2 * (p * No + k) + 1] = c * v.y - s * v.x;
  }
}

__global__ void crop_complex_kernel(const float2* __restrict__ grid, double* __restrict__ out,
                                    const float* __restrict__ sy, const float* __restrict__ sx, int Ny, int Nx,
                                    int Ky, int Kx) {
  const int64_t N = (int64_t)Ny * Nx;
  const int p = blockIdx.y;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(q / Ny), iy = (int)(q - (int64_t)ix * Ny);
    int ky = iy - Ny / 2;
    ky += ky < 0 ? Ky : 0;
    int kx = ix - Nx / 2;
    kx += kx < 0 ? Kx : 0;
    const float2 g = grid[(size_t)p * Ky * Kx + (size_t)kx * Ky + ky];
    const double sc = (double)sy[iy] * sx[ix];
    out[2 * (p * N + q)] = sc * g.x;
    out[2 * (p * N + q) + 1] = sc * g.y;
  }
}

__global__ void plane_sumsq_kernel(const float* __restrict__ x, int64_t N, double* __restrict__ out) {
  __shared__ double sh[1024];
  const int p = blockIdx.x;
  double a = 0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
    const double v = x[(size_t)p * N + i];
    a += v * v;
  }
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[p] = sh[0];
}

__global__ void plane_scale_kernel(float* __restrict__ x, int64_t N, const double* __restrict__ f) {
  const int p = blockIdx.y;
  const float s = (float)f[p];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    x[(size_t)p * N + i] *= s;
}

__global__ void vis_axpy_kernel(float2* __restrict__ y, const float2* __restrict__ x, float a, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 v = x[i];
    y[i] = make_float2(fmaf(a, v.x, y[i].x), fmaf(a, v.y, y[i].y));
  }
}

__global__ void plane_set_kernel(float* __restrict__ x, int64_t N, int np, int64_t idx, float v) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < np) x[(size_t)p * N + idx] = v;
}

__global__ void plane_max_kernel(const float* __restrict__ x, int64_t N, double* __restrict__ out) {
  __shared__ float sh[1024];
  const int p = blockIdx.x;
  float m = -INFINITY;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) m = fmaxf(m, x[(size_t)p * N + i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[p] = sh[0];
}

__global__ void plane_scale_inv_kernel(float* __restrict__ x, int64_t N, const double* __restrict__ f) {
  const int p = blockIdx.y;
  const float s = (float)(1.0 / f[p]);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    x[(size_t)p * N + i] *= s;
}

}  // namespace

void launch_vis_axpy(float2* y, const float2* x, float a, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  vis_axpy_kernel<<<nblk(n), 256, 0, s>>>(y, x, a, n);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_plane_set(float* x, int64_t N, int np, int64_t idx, float v, cudaStream_t s) {
  plane_set_kernel<<<(np + 255) / 256, 256, 0, s>>>(x, N, np, idx, v);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_plane_max(const float* x, int64_t N, int np, double* out, cudaStream_t s) {
  plane_max_kernel<<<np, 1024, 0, s>>>(x, N, out);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_plane_scale_inv(float* x, int64_t N, int np, const double* f, cudaStream_t s) {
  dim3 grid(nblk(N), np);
  plane_scale_inv_kernel<<<grid, 256, 0, s>>>(x, N, f);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_d2f(const double* in, float* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  d2f_kernel<<<nblk(n), 256, 0, s>>>(in, out, n);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_f2d(const float* in, double* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  f2d_kernel<<<nblk(n), 256, 0, s>>>(in, out, n);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_vis_gather(const double* in, float2* out, const int32_t* perm, const int64_t* ch_voff,
                       const int32_t* ch_M, int c0, int nc, int64_t maxM, int64_t host_off0, cudaStream_t s) {
  if (maxM <= 0 || nc <= 0) return;
  dim3 grid(nblk(maxM), nc);
  vis_gather_kernel<<<grid, 256, 0, s>>>(in, out, perm, ch_voff, ch_M, c0, host_off0);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_vis_scatter(const float2* in, double* out, const int32_t* perm, const int64_t* ch_voff,
                        const int32_t* ch_M, int c0, int nc, int64_t maxM, int64_t host_off0, cudaStream_t s) {
  if (maxM <= 0 || nc <= 0) return;
  dim3 grid(nblk(maxM), nc);
  vis_scatter_kernel<<<grid, 256, 0, s>>>(in, out, perm, ch_voff, ch_M, c0, host_off0);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_grid_from_matlab(const double* in, float2* out, int Ny, int Nx, int Ky, int Kx, int np,
                             cudaStream_t s) {
  dim3 grid(nblk((int64_t)Ky * Kx), np);
  grid_from_matlab_kernel<<<grid, 256, 0, s>>>(in, out, Ny, Nx, Ky, Kx);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_grid_to_matlab(const float2* in, double* out, int Ny, int Nx, int Ky, int Kx, int np,
                           cudaStream_t s) {
  dim3 grid(nblk((int64_t)Ky * Kx), np);
  grid_to_matlab_kernel<<<grid, 256, 0, s>>>(in, out, Ny, Nx, Ky, Kx);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_crop_complex(const float2* grid, double* out, const float* sy, const float* sx, int Ny, int Nx,
                         int Ky, int Kx, int np, cudaStream_t s) {
  dim3 g(nblk((int64_t)Ny * Nx), np);
  crop_complex_kernel<<<g, 256, 0, s>>>(grid, out, sy, sx, Ny, Nx, Ky, Kx);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_plane_sumsq(const float* x, int64_t N, int np, double* out, cudaStream_t s) {
  plane_sumsq_kernel<<<np, 1024, 0, s>>>(x, N, out);
  count_launch();
  FHS_LAUNCH_CHECK();
}
void launch_plane_scale(float* x, int64_t N, int np, const double* f, cudaStream_t s) {
  dim3 grid(nblk(N), np);
  plane_scale_kernel<<<grid, 256, 0, s>>>(x, N, f);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
