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

static __device__ __forceinline__ int wrap(int k, int K) {
  k %= K;
  return k < 0 ? k + K : k;
}

}  // namespace fhs
