// Complex arithmetic and min-max tap evaluation shared by the NUFFT kernels
// (measop.cu) and the visibility-gridding operator (dr.cu).
#pragma once

#include "common.cuh"
#include "minmax.h"

namespace fhs {

static __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // conj(a) * b
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
static __device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {  // a*b + c
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// Tap coefficients h_j(f) of one axis by Horner evaluation of degree-8
// polynomials in f - 1/2 (FP32, < 1e-7 relative to the FP64 construction).
template <int J>
static __device__ __forceinline__ void taps(const float (&P)[kMaxTaps][2][kPolyDegree + 1], float f, float2 (&h)[J]) {
  const float s = f - 0.5f;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    float re = P[j][0][kPolyDegree], im = P[j][1][kPolyDegree];
#pragma unroll
    for (int k = kPolyDegree - 1; k >= 0; --k) {
      re = fmaf(re, s, P[j][0][k]);
      im = fmaf(im, s, P[j][1][k]);
    }
    h[j] = make_float2(re, im);
  }
}

// The taps without their phase: h_j(f) = exp(i pi (dk - j)/K) c_j(f) with
// c_j real, so c by Horner evaluation of the real polynomials (FP32).
template <int J>
static __device__ __forceinline__ void rtaps(const float (&P)[kMaxTaps][kPolyDegree + 1], float f, float (&c)[J]) {
  const float s = f - 0.5f;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    float v = P[j][kPolyDegree];
#pragma unroll
    for (int k = kPolyDegree - 1; k >= 0; --k) v = fmaf(v, s, P[j][k]);
    c[j] = v;
  }
}

// Phase-factored taps.  With k = ks + j the unwrapped grid index of tap j
// (ks = k0 + 1, the first tap) and dk - j = om/gamma - k:
//   h_j = exp(i phi) psi(k mod K) sigma(k) c_j,
//   phi = pi (ks + f + J/2 - 1) / K = om / 2     (per visibility and axis;
//                                                 kept per visibility as
//                                                 exp(i (om_y + om_x) / 2)),
//   psi(kk) = exp(-i pi r(kk) / K), r(kk) = kk for kk < K/2, kk - K above
//                                                (per grid cell),
//   sigma(k) = +1 for -K/2 <= k < K/2, -1 outside (taps past the edge).
// The stored fractional offset f carries in its sign bit whether ks < 0
// (ks in [-K/2 - 3, K/2 - 3] for om in [-pi, pi)), which resolves the wrap.
static __device__ __forceinline__ void axis_start(float fenc, int s, int K, float& f, int& ks) {
  f = fabsf(fenc);
  ks = (__float_as_uint(fenc) >> 31) ? s - K : s;
}

// c_j <- sigma(ks + j) c_j (only visibilities within J cells of the
// +-K/2 edge of the uv plane have a tap past it)
template <int J>
static __device__ __forceinline__ void tap_signs(int ks, int K, float (&c)[J]) {
  const int h = K >> 1;
  if (ks >= -h && ks + J - 1 < h) return;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int k = ks + j;
    if (k < -h || k >= h) c[j] = -c[j];
  }
}

// psi(kk) of one axis (kk in [0, K))
static __device__ __forceinline__ float2 cell_phase(int kk, int K) {
  const int r = kk < (K >> 1) ? kk : kk - K;
  float sn, cs;
  sincospif(-(float)r / (float)K, &sn, &cs);
  return make_float2(cs, sn);
}

static __device__ __forceinline__ int wrap(int k, int K) {
  k %= K;
  return k < 0 ? k + K : k;
}

}  // namespace fhs
