// Conversion kernels between the host (MATLAB) formats and the device layout.
#pragma once

#include "common.cuh"

namespace fhs {

// double (host layout, staged on device) -> float planes
void launch_d2f(const double* in, float* out, int64_t n, cudaStream_t s);
void launch_f2d(const float* in, double* out, int64_t n, cudaStream_t s);
// complex double (interleaved) in original visibility order -> float2 sorted
void launch_vis_gather(const double* in, float2* out, const int32_t* perm, const int64_t* ch_voff,
                       const int32_t* ch_M, int c0, int nc, int64_t maxM, int64_t host_off0,
                       cudaStream_t s);
// float2 sorted -> complex double original order
void launch_vis_scatter(const float2* in, double* out, const int32_t* perm, const int64_t* ch_voff,
                        const int32_t* ch_M, int c0, int nc, int64_t maxM, int64_t host_off0,
                        cudaStream_t s);
// MATLAB-convention grid (top-left image, complex double) <-> internal grid
// (centred image): internal = rho * matlab, rho(k) = exp(i pi (ky Ny/Ky + kx Nx/Kx))
void launch_grid_from_matlab(const double* in, float2* out, int Ny, int Nx, int Ky, int Kx, int np,
                             cudaStream_t s);
void launch_grid_to_matlab(const float2* in, double* out, int Ny, int Nx, int Ky, int Kx, int np,
                           cudaStream_t s);
// complex crop of an internal grid plane times the scaling: x = s .* grid[(n - N/2) mod K]
void launch_crop_complex(const float2* grid, double* out, const float* sy, const float* sx, int Ny, int Nx,
                         int Ky, int Kx, int np, cudaStream_t s);
// per-plane sum of squares (FP64): out[p] = sum x[p][:]^2
void launch_plane_sumsq(const float* x, int64_t N, int np, double* out, cudaStream_t s);
// y <- y + a * x (float2 vectors of length n)
void launch_vis_axpy(float2* y, const float2* x, float a, int64_t n, cudaStream_t s);
// x[p][idx] = v for every plane
void launch_plane_set(float* x, int64_t N, int np, int64_t idx, float v, cudaStream_t s);
// out[p] = max x[p][:] (FP64)
void launch_plane_max(const float* x, int64_t N, int np, double* out, cudaStream_t s);
// x[p][:] /= f[p]
void launch_plane_scale_inv(float* x, int64_t N, int np, const double* f, cudaStream_t s);
// per-plane scale: x[p][:] *= f[p]
void launch_plane_scale(float* x, int64_t N, int np, const double* f, cudaStream_t s);

}  // namespace fhs
