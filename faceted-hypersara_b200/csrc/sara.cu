// SARA dictionary and weighted l21 prox on B200 (sm_100a).
//
// Replaces op_p_sp_wlt_basis / sdwt2_sara_faceting / isdwt2_sara_faceting of
// the SARA-dictionary submodule (called at imaging/imaging.m:802 and
// src/fhs/fhs_update_dual_sparsity.m:75,92) and the l21 prox of
// src/fhs/fhs_update_dual_sparsity.m:84-89 /
// src/hs/hs_update_dual_sparsity_distributed.m:41-54.
//
// Daubechies db1..db8 extremal-phase filters are computed on the host by
// spectral factorisation (Daubechies, Ten Lectures, sec. 6.1) in FP64.  One
// analysis level filters a 2-D tile along x then y (zero padding, full
// convolution, odd samples kept) and writes the four subbands in MATLAB's
// wavedec2 layout; one synthesis level is the exact adjoint.  All 8 bases and
// all channels of a level run in one launch.  The faceted transform of the
// reference produces the same coefficients as this global transform
// (segmentwise DWT, Prusa 2012), split over facets.
#include "sara.cuh"

#include <algorithm>
#include <cmath>
#include <complex>

namespace fhs {

namespace {

__constant__ float c_lo[kSaraWavelets][kSaraMaxFilter];  // Lo_D
__constant__ float c_hi[kSaraWavelets][kSaraMaxFilter];  // Hi_D

// ------------------------------------------------------------- filters
std::vector<double> poly_mul(const std::vector<double>& a, const std::vector<double>& b) {
  std::vector<double> c(a.size() + b.size() - 1, 0.0);
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < b.size(); ++j) c[i + j] += a[i] * b[j];
  return c;
}

// Roots of a real polynomial (coefficients highest degree first) by the
// Durand-Kerner iteration followed by Newton polishing.
std::vector<std::complex<double>> poly_roots(const std::vector<double>& c) {
  const int n = (int)c.size() - 1;
  std::vector<std::complex<double>> r(n);
  if (n <= 0) return r;
  auto eval = [&](std::complex<double> z) {
    std::complex<double> v = c[0];
    for (int i = 1; i <= n; ++i) v = v * z + c[i];
    return v;
  };
  auto deriv = [&](std::complex<double> z) {
    std::complex<double> v = c[0] * (double)n;
    for (int i = 1; i < n; ++i) v = v * z + c[i] * (double)(n - i);
    return v;
  };
  const std::complex<double> seed(0.4, 0.9);
  for (int i = 0; i < n; ++i) r[i] = std::pow(seed, i);
  for (int it = 0; it < 2000; ++it) {
    double delta = 0;
    for (int i = 0; i < n; ++i) {
      std::complex<double> den = c[0];
      for (int j = 0; j < n; ++j)
        if (j != i) den *= (r[i] - r[j]);
      const std::complex<double> d = eval(r[i]) / den;
      r[i] -= d;
      delta = std::max(delta, std::abs(d));
    }
    if (delta < 1e-15) break;
  }
  for (auto& z : r)
    for (int k = 0; k < 5; ++k) {
      const auto d = deriv(z);
      if (std::abs(d) > 0) z -= eval(z) / d;
    }
  return r;
}

// Extremal-phase Daubechies scaling filter with p vanishing moments, oriented
// as MATLAB's reconstruction low-pass Lo_R, normalised to sum sqrt(2).
std::vector<double> daubechies(int p) {
  std::vector<double> h;
  if (p == 1) return {1.0 / std::sqrt(2.0), 1.0 / std::sqrt(2.0)};
  // z^{p-1} P((2 - z - 1/z)/4) with P(y) = sum_k C(p-1+k, k) y^k
  const std::vector<double> base = {-0.25, 0.5, -0.25};
  std::vector<double> poly(2 * p - 1, 0.0);
  for (int k = 0; k < p; ++k) {
    double ck = 1.0;
    for (int i = 1; i <= k; ++i) ck = ck * (p - 1 + i) / i;
    std::vector<double> term = {1.0};
    for (int i = 0; i < k; ++i) term = poly_mul(term, base);
    term.resize(term.size() + (p - 1 - k), 0.0);
    const size_t off = poly.size() - term.size();
    for (size_t i = 0; i < term.size(); ++i) poly[off + i] += ck * term[i];
  }
  const auto roots = poly_roots(poly);
  std::vector<std::complex<double>> q = {1.0};
  for (const auto& z : roots) {
    if (std::abs(z) >= 1.0) continue;
    std::vector<std::complex<double>> nq(q.size() + 1, 0.0);
    for (size_t i = 0; i < q.size(); ++i) {
      nq[i] += q[i];
      nq[i + 1] -= q[i] * z;
    }
    q = nq;
  }
  h.resize(q.size());
  for (size_t i = 0; i < q.size(); ++i) h[i] = q[i].real();
  for (int i = 0; i < p; ++i) h = poly_mul(h, {1.0, 1.0});
  double sum = 0;
  for (double v : h) sum += v;
  for (double& v : h) v = v / sum * std::sqrt(2.0);
  return h;
}

bool g_filters_ready[64] = {false};

void upload_filters() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && g_filters_ready[dev]) return;
  float lo[kSaraWavelets][kSaraMaxFilter] = {};
  float hi[kSaraWavelets][kSaraMaxFilter] = {};
  for (int b = 0; b < kSaraWavelets; ++b) {
    const std::vector<double> lo_r = daubechies(b + 1);
    const int L = (int)lo_r.size();
    for (int k = 0; k < L; ++k) lo[b][k] = (float)lo_r[L - 1 - k];  // Lo_D = reverse(Lo_R)
    // Hi_D = reverse(Hi_R): Hi_D[k] = Hi_R[L-1-k] = (-1)^(L-1-k) Lo_R[k]
    for (int k = 0; k < L; ++k) hi[b][k] = (float)((((L - 1 - k) % 2) ? -1.0 : 1.0) * lo_r[k]);
  }
  FHS_CUDA(cudaMemcpyToSymbol(c_lo, lo, sizeof(lo)));
  FHS_CUDA(cudaMemcpyToSymbol(c_hi, hi, sizeof(hi)));
  if (dev < 64) g_filters_ready[dev] = true;
}

// ------------------------------------------------------------ analysis
constexpr int AT0 = 32, AT1 = 8;                 // output tile (y, x)
constexpr int AIN0 = 2 * AT0 + kSaraMaxFilter - 2;  // 78
constexpr int AIN1 = 2 * AT1 + kSaraMaxFilter - 2;  // 30

struct LevelArgs {
  int n0[kSaraWavelets], n1[kSaraWavelets];   // input sizes
  int m0[kSaraWavelets], m1[kSaraWavelets];   // output sizes
  int tiles0[kSaraWavelets], tiles[kSaraWavelets];
  int64_t in_off[kSaraWavelets];
  int64_t a_off[kSaraWavelets];
  int64_t h_off[kSaraWavelets];
  int64_t in_stride, s_stride, apx_stride;
  int first, last;   // input from x (level 1); A into coef (level J)
  float in_scale;
  int dirac;          // level 1 of the split kernel: the db1 tiles also prox the Dirac rows
  int64_t dirac_off;  // first Dirac row in a channel's coefficient vector
};

__global__ void __launch_bounds__(256) analysis_kernel(LevelArgs a, const float* __restrict__ x,
                                                       float* __restrict__ coef, float* __restrict__ apx) {
  __shared__ float sin_[AIN1][AIN0 + 1];
  __shared__ float tlo[AT1][AIN0 + 1];
  __shared__ float thi[AT1][AIN0 + 1];
  const int b = blockIdx.y;
  const int plane = blockIdx.z;
  const int tile = blockIdx.x;
  if (tile >= a.tiles[b]) return;
  const int Lf = 2 * (b + 1);
  const int n0 = a.n0[b], n1 = a.n1[b], m0 = a.m0[b], m1 = a.m1[b];
  const int tp0 = tile % a.tiles0[b], tp1 = tile / a.tiles0[b];
  const int p0s = tp0 * AT0, p1s = tp1 * AT1;
  const int i0s = 2 * p0s + 2 - Lf, i1s = 2 * p1s + 2 - Lf;
  const int IN0 = 2 * AT0 + Lf - 2, IN1 = 2 * AT1 + Lf - 2;
  const float* src = a.first ? x + (size_t)plane * a.in_stride
                             : apx + (size_t)plane * a.apx_stride + a.in_off[b];
  for (int idx = threadIdx.x; idx < IN0 * IN1; idx += blockDim.x) {
    const int l1 = idx / IN0, l0 = idx - l1 * IN0;
    const int i0 = i0s + l0, i1 = i1s + l1;
    float v = 0.f;
    if (i0 >= 0 && i0 < n0 && i1 >= 0 && i1 < n1) v = src[(size_t)i1 * n0 + i0] * a.in_scale;
    sin_[l1][l0] = v;
  }
  __syncthreads();
  // filter along x (dim 2): tlo/thi[p1][i0]
  for (int idx = threadIdx.x; idx < AT1 * IN0; idx += blockDim.x) {
    const int lp1 = idx / IN0, l0 = idx - lp1 * IN0;
    float lo = 0.f, hi = 0.f;
    for (int t = 0; t < Lf; ++t) {
      const float v = sin_[2 * lp1 + Lf - 1 - t][l0];
      lo = fmaf(c_lo[b][t], v, lo);
      hi = fmaf(c_hi[b][t], v, hi);
    }
    tlo[lp1][l0] = lo;
    thi[lp1][l0] = hi;
  }
  __syncthreads();
  const int lp0 = threadIdx.x % AT0, lp1 = threadIdx.x / AT0;
  const int p0 = p0s + lp0, p1 = p1s + lp1;
  if (lp1 < AT1 && p0 < m0 && p1 < m1) {
    float aa = 0.f, hh = 0.f, vv = 0.f, dd = 0.f;
    for (int t = 0; t < Lf; ++t) {
      const int l0 = 2 * lp0 + Lf - 1 - t;
      const float lo = tlo[lp1][l0], hi = thi[lp1][l0];
      aa = fmaf(c_lo[b][t], lo, aa);
      hh = fmaf(c_hi[b][t], lo, hh);
      vv = fmaf(c_lo[b][t], hi, vv);
      dd = fmaf(c_hi[b][t], hi, dd);
    }
    const size_t o = (size_t)p1 * m0 + p0;
    const size_t mm = (size_t)m0 * m1;
    float* cp = coef + (size_t)plane * a.s_stride + a.h_off[b];
    cp[o] = hh;
    cp[mm + o] = vv;
    cp[2 * mm + o] = dd;
    if (a.last)
      coef[(size_t)plane * a.s_stride + a.a_off[b] + o] = aa;
    else
      apx[(size_t)plane * a.apx_stride + a.a_off[b] + o] = aa;
  }
}

// Fused analysis level + l21 prox.  One CTA computes a 32 (y) x 8 (x)
// coefficient tile of one basis for every channel of a spectral group:
//  step 1: each thread takes one input row (y) of one channel, loads its
//          2*8+Lf-2 samples along x straight from global memory (coalesced
//          across threads) and filters/downsamples along x in registers; the
//          low/high outputs go to shared memory split by row parity;
//  step 2: the owner thread of each coefficient filters along y (polyphase,
//          conflict-free reads) for every channel, adds the dual v1 kept in
//          registers and applies the weighted l21 prox across the group.
// v1 is read and written once; the coefficients never reach HBM.  Grid:
// (basis, tile, group) with the basis fastest so the 8 bases of a tile share
// the input tile in L2.  The filter length is a template parameter (the
// basis index selects the instantiation) so the x-filter stays in registers.
constexpr int APH = (2 * AT0 + kSaraMaxFilter - 2 + 1) / 2;  // 39 rows per parity
constexpr int kApChunk = 16;                                 // channels staged per phase
constexpr int kApBand = 256;                                 // tiles per basis-major band of the grid

template <int MAXL, int LF, bool LAST>
__device__ __forceinline__ void analysis_prox_body(const LevelArgs& a, int b, int tile, int g,
                                                   const float* __restrict__ x, float* __restrict__ apx,
                                                   float* __restrict__ v1, const float* __restrict__ weights,
                                                   const double* __restrict__ beta, int lg,
                                                   double* __restrict__ l21_acc, float* sm, double* red) {
  constexpr int IN0 = 2 * AT0 + LF - 2, IN1 = 2 * AT1 + LF - 2;
  constexpr int CH = MAXL < kApChunk ? MAXL : kApChunk;
  // sm layout: [CH][4 (lo_e, lo_o, hi_e, hi_o)][AT1][APH]
  static_assert(IN0 <= 2 * APH, "row buffer too small");
  const int n0 = a.n0[b], n1 = a.n1[b], m0 = a.m0[b], m1 = a.m1[b];
  const int tp0 = tile % a.tiles0[b], tp1 = tile / a.tiles0[b];
  const int p0s = tp0 * AT0, p1s = tp1 * AT1;
  const int i0s = 2 * p0s + 2 - LF, i1s = 2 * p1s + 2 - LF;
  const int lp0 = threadIdx.x % AT0, lp1 = threadIdx.x / AT0;
  const int p0 = p0s + lp0, p1 = p1s + lp1;
  const bool valid = p0 < m0 && p1 < m1;
  const size_t o = (size_t)p1 * m0 + p0;
  const size_t mm = (size_t)m0 * m1;
  constexpr int NSUB = LAST ? 4 : 3;
  const int64_t off[4] = {a.h_off[b], a.h_off[b] + (int64_t)mm, a.h_off[b] + 2 * (int64_t)mm, a.a_off[b]};
  // the basis is LF / 2 - 1: the taps are compile-time constant-bank operands
  const float* lo_f = c_lo[LF / 2 - 1];
  const float* hi_f = c_hi[LF / 2 - 1];
  float w[NSUB][MAXL];
#pragma unroll
  for (int l = 0; l < MAXL; ++l) {
#pragma unroll
    for (int k = 0; k < NSUB; ++k) w[k][l] = 0.f;
    if (l < lg && valid) {
      const float* vp = v1 + ((size_t)g * lg + l) * a.s_stride;
#pragma unroll
      for (int k = 0; k < NSUB; ++k) w[k][l] = vp[off[k] + o];
    }
  }
#pragma unroll 1
  for (int c0 = 0; c0 < MAXL; c0 += CH) {
    const int nch = min(CH, lg - c0);
    if (nch <= 0) continue;
    // ---- step 1: x filtering of (row, channel) tasks
    // (interior tiles read their whole input window without bounds tests)
    const bool inside = i0s >= 0 && i0s + IN0 <= n0 && i1s >= 0 && i1s + IN1 <= n1;
    const float scale = a.in_scale;
    for (int task = threadIdx.x; task < IN0 * nch; task += blockDim.x) {
      const int r = task % IN0, lc = task / IN0;
      const size_t plane = (size_t)g * lg + c0 + lc;
      const float* src = a.first ? x + plane * a.in_stride : apx + plane * a.apx_stride + a.in_off[b];
      const int i0 = i0s + r;
      float v[IN1];
      if (inside) {
        const float* row = src + (ptrdiff_t)i1s * n0 + i0;
#pragma unroll
        for (int c = 0; c < IN1; ++c) v[c] = row[c * n0];
      } else {
        const bool rin = i0 >= 0 && i0 < n0;
#pragma unroll
        for (int c = 0; c < IN1; ++c) {
          const int i1 = i1s + c;
          v[c] = (rin && i1 >= 0 && i1 < n1) ? src[(size_t)i1 * n0 + i0] : 0.f;
        }
      }
      float* base = sm + (size_t)lc * 4 * AT1 * APH;
      const int par = r & 1, rh = r >> 1;
#pragma unroll
      for (int q = 0; q < AT1; ++q) {
        float lo = 0.f, hi = 0.f;
#pragma unroll
        for (int t = 0; t < LF; ++t) {
          lo = fmaf(lo_f[t], v[2 * q + LF - 1 - t], lo);
          hi = fmaf(hi_f[t], v[2 * q + LF - 1 - t], hi);
        }
        base[(0 + par) * AT1 * APH + q * APH + rh] = lo * scale;
        base[(2 + par) * AT1 * APH + q * APH + rh] = hi * scale;
      }
    }
    __syncthreads();
    // ---- step 2: y filtering by the owner of each coefficient
    if constexpr (MAXL <= kApChunk) {
      // channels unrolled inside the taps: the filter sums accumulate straight
      // into the dual w[][l] (compile-time register indices, no selects)
      float aa[LAST ? 1 : MAXL];
#pragma unroll
      for (int l = 0; l < (LAST ? 1 : MAXL); ++l) aa[l] = 0.f;
      const float* col = sm + lp1 * APH;
#pragma unroll
      for (int t = 0; t < LF; ++t) {
        const int r = 2 * lp0 + LF - 1 - t;   // parity of r is that of LF - 1 - t
        const int par = (LF - 1 - t) & 1, rh = r >> 1;
#pragma unroll
        for (int l = 0; l < MAXL; ++l) {
          if (l < nch) {
            const float* base = col + (size_t)l * 4 * AT1 * APH;
            const float lo = base[(0 + par) * AT1 * APH + rh];
            const float hi = base[(2 + par) * AT1 * APH + rh];
            w[0][l] = fmaf(hi_f[t], lo, w[0][l]);
            w[1][l] = fmaf(lo_f[t], hi, w[1][l]);
            w[2][l] = fmaf(hi_f[t], hi, w[2][l]);
            if constexpr (LAST)
              w[NSUB - 1][l] = fmaf(lo_f[t], lo, w[NSUB - 1][l]);
            else
              aa[l] = fmaf(lo_f[t], lo, aa[l]);
          }
        }
      }
      if constexpr (!LAST) {
        if (valid) {
#pragma unroll
          for (int l = 0; l < MAXL; ++l)
            if (l < nch) apx[((size_t)g * lg + l) * a.apx_stride + a.a_off[b] + o] = aa[l];
        }
      }
      __syncthreads();
      continue;
    }
#pragma unroll 1
    for (int lc = 0; lc < CH; ++lc) {
      const int l = c0 + lc;
      if (lc < nch) {
        const float* base = sm + (size_t)lc * 4 * AT1 * APH + lp1 * APH;
        float aa = 0.f, hh = 0.f, vv = 0.f, dd = 0.f;
#pragma unroll
        for (int t = 0; t < LF; ++t) {
          const int r = 2 * lp0 + LF - 1 - t;
          const int par = r & 1, rh = r >> 1;
          const float lo = base[(0 + par) * AT1 * APH + rh];
          const float hi = base[(2 + par) * AT1 * APH + rh];
          aa = fmaf(lo_f[t], lo, aa);
          hh = fmaf(hi_f[t], lo, hh);
          vv = fmaf(lo_f[t], hi, vv);
          dd = fmaf(hi_f[t], hi, dd);
        }
#pragma unroll
        for (int ll = 0; ll < MAXL; ++ll)
          if (ll == l) {
            w[0][ll] += hh;
            w[1][ll] += vv;
            w[2][ll] += dd;
            if constexpr (LAST) w[NSUB - 1][ll] += aa;
          }
        if (!LAST && valid) apx[((size_t)g * lg + l) * a.apx_stride + a.a_off[b] + o] = aa;
      }
    }
    __syncthreads();
  }
  double l21 = 0.0;
  if (valid) {
    const float bt = (float)beta[g];
    const float* wg = weights + (size_t)g * a.s_stride;
#pragma unroll
    for (int k = 0; k < NSUB; ++k) {
      float ss = 0.f;
#pragma unroll
      for (int l = 0; l < MAXL; ++l)
        if (l < lg) ss = fmaf(w[k][l], w[k][l], ss);
      const float l2 = sqrtf(ss);
      l21 += l2;
      const float soft = fmaxf(l2 - bt * wg[off[k] + o], 0.f) / (l2 + 2.220446049250313e-16f);
#pragma unroll
      for (int l = 0; l < MAXL; ++l)
        if (l < lg) v1[((size_t)g * lg + l) * a.s_stride + off[k] + o] = w[k][l] - soft * w[k][l];
    }
  }
  if (l21_acc) {
    for (int sh = 16; sh > 0; sh >>= 1) l21 += __shfl_down_sync(0xffffffffu, l21, sh);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l21;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < 8; ++i) t += red[i];
      atomicAdd(l21_acc + g, t);
    }
  }
}

template <int MAXL>
__global__ void __launch_bounds__(256, (MAXL > 16 ? 1 : 2)) analysis_prox_kernel(LevelArgs a, const float* __restrict__ x,
                                                            float* __restrict__ apx, float* __restrict__ v1,
                                                            const float* __restrict__ weights,
                                                            const double* __restrict__ beta, int lg,
                                                            double* __restrict__ l21_acc) {
  extern __shared__ float sm_ap[];
  __shared__ double red[8];
  // blockIdx.x = (band, basis, tile in band): the CTAs resident together run
  // one basis (one code path), and the 8 bases of a band of kApBand tiles
  // follow each other while its input is still in L2
  const int band = blockIdx.x / (kSaraWavelets * kApBand);
  const int rem = blockIdx.x - band * (kSaraWavelets * kApBand);
  const int b = rem / kApBand, tile = band * kApBand + rem % kApBand, g = blockIdx.y;
  if (tile >= a.tiles[b]) return;
  if (a.last) {
    switch (b) {
#define FHS_C(BB, LFV) \
  case BB: analysis_prox_body<MAXL, LFV, true>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red); break;
      FHS_C(0, 2) FHS_C(1, 4) FHS_C(2, 6) FHS_C(3, 8) FHS_C(4, 10) FHS_C(5, 12) FHS_C(6, 14) FHS_C(7, 16)
#undef FHS_C
    }
  } else {
    switch (b) {
#define FHS_C(BB, LFV) \
  case BB: analysis_prox_body<MAXL, LFV, false>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red); break;
      FHS_C(0, 2) FHS_C(1, 4) FHS_C(2, 6) FHS_C(3, 8) FHS_C(4, 10) FHS_C(5, 12) FHS_C(6, 14) FHS_C(7, 16)
#undef FHS_C
    }
  }
}

template <int MAXL>
size_t analysis_prox_smem() {
  constexpr int CH = MAXL < kApChunk ? MAXL : kApChunk;
  return (size_t)CH * 4 * AT1 * APH * sizeof(float);
}

template <int MAXL>
void launch_analysis_prox(dim3 grid, cudaStream_t s, const LevelArgs& a, const float* x, float* apx, float* v1,
                          const float* weights, const double* beta, int lg, double* l21_acc) {
  const size_t smem = analysis_prox_smem<MAXL>();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev < 64 && !attr[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(analysis_prox_kernel<MAXL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    attr[dev] = true;
  }
  analysis_prox_kernel<MAXL><<<grid, 256, smem, s>>>(a, x, apx, v1, weights, beta, lg, l21_acc);
}

// The same fused level for groups of at most 16 channels with two threads per
// coefficient position (512 threads per 32 x 8 tile): thread branch 0 takes
// the y-low-pass of the x-low rows (A) and their y-high-pass (H), branch 1
// the y-low and y-high passes of the x-high rows (V, D).  Each thread holds
// 2 subbands x 16 channels of the dual, loaded after the x filtering, so the
// kernel fits 64 registers and 2 CTAs per SM (32 warps).
constexpr int kApSplitThreads = 2 * AT0 * AT1;

// step 1 of the split kernel: (input row, channel) tasks filter and
// downsample along x (all 512 threads) into sm [channel][lo e/o, hi e/o][AT1][APH]
template <int LF>
__device__ __forceinline__ void ap_split_xfilter(const LevelArgs& a, int b, int tile, int g,
                                                 const float* __restrict__ x, const float* __restrict__ apx, int lg,
                                                 float* sm) {
  constexpr int IN0 = 2 * AT0 + LF - 2, IN1 = 2 * AT1 + LF - 2;
  constexpr int B = LF / 2 - 1;
  static_assert(IN0 <= 2 * APH, "row buffer too small");
  const float* lo_f = c_lo[B];
  const float* hi_f = c_hi[B];
  const int n0 = a.n0[b], n1 = a.n1[b];
  const int tp0 = tile % a.tiles0[b], tp1 = tile / a.tiles0[b];
  const int i0s = 2 * tp0 * AT0 + 2 - LF, i1s = 2 * tp1 * AT1 + 2 - LF;
  const bool inside = i0s >= 0 && i0s + IN0 <= n0 && i1s >= 0 && i1s + IN1 <= n1;
  const float scale = a.in_scale;
  for (int task = threadIdx.x; task < IN0 * lg; task += kApSplitThreads) {
    const int r = task % IN0, lc = task / IN0;
    const size_t plane = (size_t)g * lg + lc;
    const float* src = a.first ? x + plane * a.in_stride : apx + plane * a.apx_stride + a.in_off[b];
    const int i0 = i0s + r;
    float v[IN1];
    if (inside) {
      const float* row = src + (ptrdiff_t)i1s * n0 + i0;
#pragma unroll
      for (int c = 0; c < IN1; ++c) v[c] = row[c * n0];
    } else {
      const bool rin = i0 >= 0 && i0 < n0;
#pragma unroll
      for (int c = 0; c < IN1; ++c) {
        const int i1 = i1s + c;
        v[c] = (rin && i1 >= 0 && i1 < n1) ? src[(size_t)i1 * n0 + i0] : 0.f;
      }
    }
    float* base = sm + (size_t)lc * 4 * AT1 * APH;
    const int par = r & 1, rh = r >> 1;
#pragma unroll
    for (int q = 0; q < AT1; ++q) {
      float lo = 0.f, hi = 0.f;
#pragma unroll
      for (int t = 0; t < LF; ++t) {
        lo = fmaf(lo_f[t], v[2 * q + LF - 1 - t], lo);
        hi = fmaf(hi_f[t], v[2 * q + LF - 1 - t], hi);
      }
      base[(0 + par) * AT1 * APH + q * APH + rh] = lo * scale;
      base[(2 + par) * AT1 * APH + q * APH + rh] = hi * scale;
    }
  }
}

// steps 2-3 of the split kernel for branch BR: the dual of the branch's two
// subbands, the y filtering accumulated into it, the weighted l21 prox
template <int MAXL, int LF, bool LAST, int BR>
__device__ __forceinline__ void ap_split_tail(const LevelArgs& a, int b, int tile, int g, const float* __restrict__ x,
                                              float* __restrict__ apx,
                                              float* __restrict__ v1, const float* __restrict__ weights,
                                              const double* __restrict__ beta, int lg,
                                              double* __restrict__ l21_acc, const float* sm, double* red) {
  constexpr int B = LF / 2 - 1;
  static_assert(MAXL <= kApChunk, "one staging round");
  // the two y filters of this branch: f0 -> subband k0, f1 -> subband k1
  // (branch 0: H = hi(y) lo(x), A = lo(y) lo(x); branch 1: V = lo(y) hi(x), D = hi(y) hi(x))
  const float* f0 = BR == 0 ? c_hi[B] : c_lo[B];
  const float* f1 = BR == 0 ? c_lo[B] : c_hi[B];
  const int m0 = a.m0[b], m1 = a.m1[b];
  const int tp0 = tile % a.tiles0[b], tp1 = tile / a.tiles0[b];
  const int pos = threadIdx.x % (AT0 * AT1);
  const int lp0 = pos % AT0, lp1 = pos / AT0;
  const int p0 = tp0 * AT0 + lp0, p1 = tp1 * AT1 + lp1;
  const bool valid = p0 < m0 && p1 < m1;
  const size_t o = (size_t)p1 * m0 + p0;
  const size_t mm = (size_t)m0 * m1;
  // subbands of this branch in the coefficient vector: H, V, D at h_off + k mm, A at a_off
  const int64_t off0 = a.h_off[b] + (BR == 0 ? 0 : (int64_t)mm);
  const int64_t off1 = BR == 0 ? a.a_off[b] : a.h_off[b] + 2 * (int64_t)mm;
  constexpr bool PROX1 = BR == 1 || LAST;   // A is a prox subband only at the last level
  const int nch = lg;
  float w0[MAXL], w1[MAXL];
#pragma unroll
  for (int l = 0; l < MAXL; ++l) {
    w0[l] = 0.f;
    w1[l] = 0.f;
    if (l < nch && valid) {
      const float* vp = v1 + ((size_t)g * lg + l) * a.s_stride + o;
      w0[l] = vp[off0];
      if (PROX1) w1[l] = vp[off1];
    }
  }
  __syncthreads();   // step 1 complete
  // taps in pairs (2u, 2u + 1): rows 2 lp0 + LF - 1 - t of odd then even
  // parity share the half-row index lp0 + LF / 2 - 1 - u; the pair loop is
  // not unrolled (compact code: all bases and branches of a launch share the
  // instruction cache), the channels are
  const float* col = sm + (BR == 0 ? 0 : 2) * AT1 * APH + lp1 * APH + lp0 + LF / 2 - 1;
#pragma unroll 1
  for (int u = 0; u < LF / 2; ++u) {
    const float f0o = f0[2 * u], f0e = f0[2 * u + 1], f1o = f1[2 * u], f1e = f1[2 * u + 1];
    const float* cu = col - u;
#pragma unroll
    for (int l = 0; l < MAXL; ++l) {
      if (l < nch) {
        const float so = cu[(size_t)l * 4 * AT1 * APH + AT1 * APH];   // odd rows
        const float se = cu[(size_t)l * 4 * AT1 * APH];               // even rows
        w0[l] = fmaf(f0o, so, fmaf(f0e, se, w0[l]));
        w1[l] = fmaf(f1o, so, fmaf(f1e, se, w1[l]));
      }
    }
  }
  if (!PROX1 && valid) {   // coarser level: A goes to the approximation scratch
#pragma unroll
    for (int l = 0; l < MAXL; ++l)
      if (l < nch) apx[((size_t)g * lg + l) * a.apx_stride + a.a_off[b] + o] = w1[l];
  }
  double l21 = 0.0;
  if (valid) {
    const float bt = (float)beta[g];
    const float* wg = weights + (size_t)g * a.s_stride + o;
    auto prox = [&](float(&w)[MAXL], int64_t off) {
      float ss = 0.f;
#pragma unroll
      for (int l = 0; l < MAXL; ++l)
        if (l < nch) ss = fmaf(w[l], w[l], ss);
      const float l2 = sqrtf(ss);
      l21 += l2;
      const float soft = fmaxf(l2 - bt * wg[off], 0.f) / (l2 + 2.220446049250313e-16f);
      float* dst = v1 + (size_t)g * lg * a.s_stride + off + o;
#pragma unroll
      for (int l = 0; l < MAXL; ++l)
        if (l < nch) dst[(size_t)l * a.s_stride] = w[l] - soft * w[l];
    };
    prox(w0, off0);
    if (PROX1) prox(w1, off1);
  }
  if constexpr (LF == 2) {
    // level 1, db1: a tile's input block (64 rows x 16 columns, no halo) is
    // a partition of the image, so these CTAs also take the Dirac rows of
    // their pixels (coefficients xhat / 3), two pixels per thread
    if (a.dirac) {
      const float bt = (float)beta[g];
      const int n0i = a.n0[0], n1i = a.n1[0];
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        const int k = threadIdx.x + h * kApSplitThreads;
        const int r = 2 * AT0 * tp0 + (k & (2 * AT0 - 1)), c = 2 * AT1 * tp1 + k / (2 * AT0);
        if (r >= n0i || c >= n1i) continue;
        const int64_t pix = (int64_t)c * n0i + r, i = a.dirac_off + pix;
        float w[MAXL];
        float ss = 0.f;
#pragma unroll
        for (int l = 0; l < MAXL; ++l) {
          w[l] = 0.f;
          if (l < nch) {
            const size_t plane = (size_t)g * lg + l;
            w[l] = v1[plane * a.s_stride + i] + __ldg(x + plane * a.in_stride + pix) * (1.f / 3.f);
            ss = fmaf(w[l], w[l], ss);
          }
        }
        const float l2 = sqrtf(ss);
        l21 += l2;
        const float soft = fmaxf(l2 - bt * weights[(size_t)g * a.s_stride + i], 0.f) / (l2 + 2.220446049250313e-16f);
#pragma unroll
        for (int l = 0; l < MAXL; ++l)
          if (l < nch) v1[((size_t)g * lg + l) * a.s_stride + i] = w[l] - soft * w[l];
      }
    }
  }
  if (l21_acc) {
    for (int sh = 16; sh > 0; sh >>= 1) l21 += __shfl_down_sync(0xffffffffu, l21, sh);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l21;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < kApSplitThreads / 32; ++i) t += red[i];
      atomicAdd(l21_acc + g, t);
    }
  }
}

template <int MAXL>
__global__ void __launch_bounds__(kApSplitThreads, 2) analysis_prox_split_kernel(
    LevelArgs a, const float* __restrict__ x, float* __restrict__ apx, float* __restrict__ v1,
    const float* __restrict__ weights, const double* __restrict__ beta, int lg, double* __restrict__ l21_acc) {
  extern __shared__ float sm_ap[];
  __shared__ double red[kApSplitThreads / 32];
  const int band = blockIdx.x / (kSaraWavelets * kApBand);
  const int rem = blockIdx.x - band * (kSaraWavelets * kApBand);
  const int b = rem / kApBand, tile = band * kApBand + rem % kApBand, g = blockIdx.y;
  if (tile >= a.tiles[b]) return;
  const int br = threadIdx.x / (AT0 * AT1);   // warp-uniform
#define FHS_C(BB, LFV)                                                                                  \
  case BB:                                                                                              \
    ap_split_xfilter<LFV>(a, b, tile, g, x, apx, lg, sm_ap);                                            \
    if (a.last) {                                                                                       \
      if (br == 0)                                                                                      \
        ap_split_tail<MAXL, LFV, true, 0>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red);  \
      else                                                                                              \
        ap_split_tail<MAXL, LFV, true, 1>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red);  \
    } else {                                                                                            \
      if (br == 0)                                                                                      \
        ap_split_tail<MAXL, LFV, false, 0>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red); \
      else                                                                                              \
        ap_split_tail<MAXL, LFV, false, 1>(a, b, tile, g, x, apx, v1, weights, beta, lg, l21_acc, sm_ap, red); \
    }                                                                                                   \
    break;
  switch (b) { FHS_C(0, 2) FHS_C(1, 4) FHS_C(2, 6) FHS_C(3, 8) FHS_C(4, 10) FHS_C(5, 12) FHS_C(6, 14) FHS_C(7, 16) }
#undef FHS_C
}

template <int MAXL>
void launch_analysis_prox_split(dim3 grid, cudaStream_t s, const LevelArgs& a, const float* x, float* apx,
                                float* v1, const float* weights, const double* beta, int lg, double* l21_acc) {
  const size_t smem = analysis_prox_smem<MAXL>();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev < 64 && !attr[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(analysis_prox_split_kernel<MAXL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    attr[dev] = true;
  }
  analysis_prox_split_kernel<MAXL><<<grid, kApSplitThreads, smem, s>>>(a, x, apx, v1, weights, beta, lg, l21_acc);
}

// ----------------------------------------------------------- synthesis
// One synthesis level is the adjoint of an analysis level: with an even tile
// start, the output pair (2k, 2k+1) along an axis draws on the same LF/2
// coefficients c[k..k+LF/2-1]:
//   out[2k] = sum_j c[k+j] f[2j+1],   out[2k+1] = sum_j c[k+j] f[2j]
// (f = Lo_D or Hi_D, t = 2p + 1 - i of the full-convolution adjoint).  A CTA
// owns a 64 (y) x 32 (x) output tile: it stages the four subbands' coefficient
// window (32 + LF/2 - 1 rows x 16 + LF/2 - 1 columns), filters along y (one
// thread per column and output pair) into shared memory, then along x (one
// thread per output row, 8 output columns in registers).  The filter length
// is a template parameter selected per basis, so both filters live in
// registers.  Final level: the CTA loops over the 8 bases, accumulating in
// registers, and adds the Dirac part; coarser levels write one basis each.
constexpr int SY = 64, SX = 32;                         // output tile (y, x)
constexpr int SRY = SY / 2 + kSaraMaxFilter / 2 - 1;    // 39 coefficient rows
constexpr int SRX = SX / 2 + kSaraMaxFilter / 2 - 1;    // 23 coefficient columns
constexpr int SRYP = SRY + 1;                           // row pitch of the window

struct SynArgs {
  int m0[kSaraWavelets], m1[kSaraWavelets];    // coefficient sizes (level j)
  int n0[kSaraWavelets], n1[kSaraWavelets];    // output sizes (level j-1)
  int tiles0[kSaraWavelets], tiles[kSaraWavelets];
  int64_t a_off[kSaraWavelets];                // A_j (coef if from_coef, else apx)
  int64_t h_off[kSaraWavelets];                // H_j in coef
  int64_t out_off[kSaraWavelets];              // level j-1 approximation in apx
  int64_t s_stride, apx_stride, out_stride;
  int a_from_coef;
  int final_level;                             // j == 1: sum bases + Dirac into out
  int64_t dirac_off;
  float alpha;
};

struct SynSmem {
  float sub[2][4][SRX][SRYP];  // A, H, V, D coefficient windows, double-buffered
  float tl[SRX][SY];           // y-filtered low  (A lo + H hi)
  float th[SRX][SY];           // y-filtered high (V lo + D hi)
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 4 : 0;  // 0 source bytes: the destination is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Starts the asynchronous copy of basis b's coefficient window for the tile
// at (I0s, I1s) into buffer buf (zeros outside the coefficient arrays).
__device__ __forceinline__ void syn_window(const SynArgs& a, int b, int plane, const float* __restrict__ coef,
                                           const float* __restrict__ apx, int I0s, int I1s, SynSmem& S, int buf) {
  const int H = b + 1;  // LF / 2
  const int RY = SY / 2 + H - 1, RX = SX / 2 + H - 1;
  const int m0 = a.m0[b], m1 = a.m1[b];
  const int P0s = I0s / 2, P1s = I1s / 2;
  const float* A = (a.a_from_coef ? coef + (size_t)plane * a.s_stride : apx + (size_t)plane * a.apx_stride) +
                   a.a_off[b];
  const float* Hc = coef + (size_t)plane * a.s_stride + a.h_off[b];
  const size_t mm = (size_t)m0 * m1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int l1 = warp; l1 < RX; l1 += 8) {  // one window column per warp, rows across lanes
    const int p1 = P1s + l1;
    for (int l0 = lane; l0 < RY; l0 += 32) {
      const int p0 = P0s + l0;
      const bool in = p0 < m0 && p1 < m1;
      const size_t o = in ? (size_t)p1 * m0 + p0 : 0;
      cp_async4(&S.sub[buf][0][l1][l0], A + o, in);
      cp_async4(&S.sub[buf][1][l1][l0], Hc + o, in);
      cp_async4(&S.sub[buf][2][l1][l0], Hc + mm + o, in);
      cp_async4(&S.sub[buf][3][l1][l0], Hc + 2 * mm + o, in);
    }
  }
  cp_async_commit();
}

// Adds basis b's synthesis (window in buffer buf, already resident) to
// acc[q] (output row threadIdx.x % 64, column 8 (threadIdx.x / 64) + q).
template <int LF>
__device__ __forceinline__ void syn_basis(int b, SynSmem& S, int buf, float acc[8]) {
  constexpr int H = LF / 2;
  constexpr int RX = SX / 2 + H - 1;
  float lo[LF], hi[LF];
#pragma unroll
  for (int t = 0; t < LF; ++t) {
    lo[t] = c_lo[b][t];
    hi[t] = c_hi[b][t];
  }
  // along y: task = (column l1, output pairs k, k + 1), k even and fastest;
  // the two pairs share H - 1 of their H + 1 coefficient rows
  for (int task = threadIdx.x; task < RX * (SY / 4); task += blockDim.x) {
    const int l1 = task / (SY / 4), k = 2 * (task - l1 * (SY / 4));
    float le0 = 0.f, lo0 = 0.f, he0 = 0.f, ho0 = 0.f, le1 = 0.f, lo1 = 0.f, he1 = 0.f, ho1 = 0.f;
#pragma unroll
    for (int j = 0; j <= H; ++j) {
      const float ca = S.sub[buf][0][l1][k + j], ch = S.sub[buf][1][l1][k + j];
      const float cv = S.sub[buf][2][l1][k + j], cd = S.sub[buf][3][l1][k + j];
      if (j < H) {   // tap j of pair k
        le0 = fmaf(ca, lo[2 * j + 1], fmaf(ch, hi[2 * j + 1], le0));
        lo0 = fmaf(ca, lo[2 * j], fmaf(ch, hi[2 * j], lo0));
        he0 = fmaf(cv, lo[2 * j + 1], fmaf(cd, hi[2 * j + 1], he0));
        ho0 = fmaf(cv, lo[2 * j], fmaf(cd, hi[2 * j], ho0));
      }
      if (j > 0) {   // tap j - 1 of pair k + 1
        le1 = fmaf(ca, lo[2 * j - 1], fmaf(ch, hi[2 * j - 1], le1));
        lo1 = fmaf(ca, lo[2 * j - 2], fmaf(ch, hi[2 * j - 2], lo1));
        he1 = fmaf(cv, lo[2 * j - 1], fmaf(cd, hi[2 * j - 1], he1));
        ho1 = fmaf(cv, lo[2 * j - 2], fmaf(cd, hi[2 * j - 2], ho1));
      }
    }
    *reinterpret_cast<float4*>(&S.tl[l1][2 * k]) = make_float4(le0, lo0, le1, lo1);
    *reinterpret_cast<float4*>(&S.th[l1][2 * k]) = make_float4(he0, ho0, he1, ho1);
  }
  __syncthreads();
  // along x: output row i0, pairs m = 4 grp + q (columns 2m, 2m+1)
  const int i0 = threadIdx.x % SY, grp = threadIdx.x / SY;
  float cl[H + 3], ch[H + 3];
#pragma unroll
  for (int c = 0; c < H + 3; ++c) {
    cl[c] = S.tl[4 * grp + c][i0];
    ch[c] = S.th[4 * grp + c][i0];
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float e = 0.f, o = 0.f;
#pragma unroll
    for (int j = 0; j < H; ++j) {
      e = fmaf(cl[q + j], lo[2 * j + 1], fmaf(ch[q + j], hi[2 * j + 1], e));
      o = fmaf(cl[q + j], lo[2 * j], fmaf(ch[q + j], hi[2 * j], o));
    }
    acc[2 * q] += e;
    acc[2 * q + 1] += o;
  }
}

__device__ __forceinline__ void syn_dispatch(int b, SynSmem& S, int buf, float acc[8]) {
  switch (b) {
    case 0: syn_basis<2>(b, S, buf, acc); break;
    case 1: syn_basis<4>(b, S, buf, acc); break;
    case 2: syn_basis<6>(b, S, buf, acc); break;
    case 3: syn_basis<8>(b, S, buf, acc); break;
    case 4: syn_basis<10>(b, S, buf, acc); break;
    case 5: syn_basis<12>(b, S, buf, acc); break;
    case 6: syn_basis<14>(b, S, buf, acc); break;
    default: syn_basis<16>(b, S, buf, acc); break;
  }
}

// Final level: the window of basis b+1 is in flight while basis b is filtered.
// Buffer (b+1)&1 was last read by basis b-1's y pass, which every thread has
// finished at basis b-1's second barrier; tl/th are rewritten by basis b's y
// pass only after its first barrier, which follows basis b-1's x pass.
__global__ void __launch_bounds__(256, 4) synthesis_kernel(SynArgs a, const float* __restrict__ coef,
                                                        float* __restrict__ apx, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char syn_smem[];
  SynSmem& S = *reinterpret_cast<SynSmem*>(syn_smem);
  const int plane = blockIdx.z;
  const int tile = blockIdx.x;
  const int i0 = threadIdx.x % SY, grp = threadIdx.x / SY;
  float acc[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) acc[q] = 0.f;
  if (!a.final_level) {
    const int b = blockIdx.y;
    if (tile >= a.tiles[b]) return;
    const int ti0 = tile % a.tiles0[b], ti1 = tile / a.tiles0[b];
    const int I0s = ti0 * SY, I1s = ti1 * SX;
    syn_window(a, b, plane, coef, apx, I0s, I1s, S, 0);
    cp_async_wait<0>();
    __syncthreads();
    syn_dispatch(b, S, 0, acc);
    const int n0 = a.n0[b], n1 = a.n1[b];
    float* dst = apx + (size_t)plane * a.apx_stride + a.out_off[b];
    if (I0s + i0 < n0) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i1 = I1s + 8 * grp + q;
        if (i1 < n1) dst[(size_t)i1 * n0 + I0s + i0] = acc[q];
      }
    }
    return;
  }
  // final level: all bases share the output size (the image)
  const int n0 = a.n0[0], n1 = a.n1[0];
  if (tile >= a.tiles[0]) return;
  const int ti0 = tile % a.tiles0[0], ti1 = tile / a.tiles0[0];
  const int I0s = ti0 * SY, I1s = ti1 * SX;
  syn_window(a, 0, plane, coef, apx, I0s, I1s, S, 0);
#pragma unroll 1
  for (int b = 0; b < kSaraWavelets; ++b) {
    if (b + 1 < kSaraWavelets) {
      syn_window(a, b + 1, plane, coef, apx, I0s, I1s, S, (b + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    syn_dispatch(b, S, b & 1, acc);
  }
  if (I0s + i0 < n0) {
    const float* dirac = coef + (size_t)plane * a.s_stride + a.dirac_off;
    float* dst = out + (size_t)plane * a.out_stride;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i1 = I1s + 8 * grp + q;
      if (i1 < n1) {
        const size_t o = (size_t)i1 * n0 + I0s + i0;
        dst[o] = a.alpha * (acc[q] + dirac[o]);
      }
    }
  }
}

// ------------------------------------------------------------- prox
// DIRAC: every row lies in the Dirac part (coefficients xhat/3, no branch, so
// the loads of all channels issue together).
template <int MAXL, bool DIRAC>
__global__ void __launch_bounds__(256) l21_prox_kernel(float* __restrict__ v1, const float* __restrict__ coef,
                                                       const float* __restrict__ xhat,
                                                       const float* __restrict__ weights,
                                                       const double* __restrict__ beta, int64_t s,
                                                       int64_t dirac_off, int64_t npix, int lg,
                                                       double* __restrict__ l21_partials, int64_t i_begin,
                                                       double* __restrict__ l21_acc) {
  const int g = blockIdx.y;
  const float bt = (float)beta[g];
  const float* wg = weights + (size_t)g * s;
  double l21 = 0.0;
  for (int64_t i = i_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s;
       i += (int64_t)gridDim.x * blockDim.x) {
    float w[MAXL];
    float ss = 0.f;
#pragma unroll
    for (int l = 0; l < MAXL; ++l) {
      if (l < lg) {
        const size_t plane = (size_t)g * lg + l;
        const float c = (DIRAC || i >= dirac_off) ? xhat[plane * npix + (i - dirac_off)] * (1.f / 3.f)
                                                  : coef[plane * s + i];
        w[l] = v1[plane * s + i] + c;
        ss = fmaf(w[l], w[l], ss);
      }
    }
    const float l2 = sqrtf(ss);
    l21 += l2;
    const float soft = fmaxf(l2 - bt * wg[i], 0.f) / (l2 + 2.220446049250313e-16f);
#pragma unroll
    for (int l = 0; l < MAXL; ++l)
      if (l < lg) v1[((size_t)g * lg + l) * s + i] = w[l] - soft * w[l];
  }
  if (l21_partials || l21_acc) {
    __shared__ double red[256];
    red[threadIdx.x] = l21;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
      if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (l21_partials) l21_partials[(size_t)g * gridDim.x + blockIdx.x] = red[0];
      if (l21_acc) atomicAdd(l21_acc + g, red[0]);
    }
  }
}

__global__ void row_norms_kernel(const float* __restrict__ coef, const float* __restrict__ x, int64_t s,
                                 int64_t dirac_off, int64_t npix, int lg, float* __restrict__ out) {
  const int g = blockIdx.y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (int64_t)gridDim.x * blockDim.x) {
    double ss = 0.0;
    for (int l = 0; l < lg; ++l) {
      const size_t plane = (size_t)g * lg + l;
      const float c = i < dirac_off ? coef[plane * s + i] : x[plane * npix + (i - dirac_off)] * (1.f / 3.f);
      ss += (double)c * c;
    }
    out[(size_t)g * s + i] = (float)sqrt(ss);
  }
}

__global__ void dirac_kernel(const float* __restrict__ x, float* __restrict__ coef, int64_t s, int64_t off,
                             int64_t npix) {
  const int plane = blockIdx.y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (int64_t)gridDim.x * blockDim.x)
    coef[(size_t)plane * s + off + i] = x[(size_t)plane * npix + i] * (1.f / 3.f);
}

int nblk(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

}  // namespace

SaraPlan sara_plan(int Ny, int Nx, int J) {
  FHS_CHECK(Ny > 0 && Nx > 0, FHS_ERR_INVALID_ARG, "bad image size");
  FHS_CHECK(J >= 1 && J <= kSaraMaxLevel, FHS_ERR_UNSUPPORTED, "nlevel must be in [1, 8]");
  SaraPlan p;
  p.Ny = Ny;
  p.Nx = Nx;
  p.J = J;
  int64_t pos = 0, apos = 0;
  for (int b = 0; b < kSaraWavelets; ++b) {
    const int Lf = 2 * (b + 1);
    p.n0[b][0] = Ny;
    p.n1[b][0] = Nx;
    for (int j = 1; j <= J; ++j) {
      p.n0[b][j] = (p.n0[b][j - 1] + Lf - 1) / 2;
      p.n1[b][j] = (p.n1[b][j - 1] + Lf - 1) / 2;
    }
    p.boff[b] = pos;
    p.offA[b] = pos;
    pos += (int64_t)p.n0[b][J] * p.n1[b][J];
    for (int j = J; j >= 1; --j) {
      p.offH[b][j] = pos;
      pos += 3 * (int64_t)p.n0[b][j] * p.n1[b][j];
    }
    for (int j = 1; j < J; ++j) {
      p.apx_off[b][j] = apos;
      apos += (int64_t)p.n0[b][j] * p.n1[b][j];
    }
  }
  p.boff[kSaraWavelets] = pos;
  pos += (int64_t)Ny * Nx;
  p.s = pos;
  p.apx_total = std::max<int64_t>(apos, 1);
  return p;
}

void sara_analysis(const SaraPlan& p, const float* x, float* coef, float* apx, int np, cudaStream_t s) {
  upload_filters();
  for (int j = 1; j <= p.J; ++j) {
    LevelArgs a{};
    int maxt = 0;
    for (int b = 0; b < kSaraWavelets; ++b) {
      a.n0[b] = p.n0[b][j - 1];
      a.n1[b] = p.n1[b][j - 1];
      a.m0[b] = p.n0[b][j];
      a.m1[b] = p.n1[b][j];
      a.tiles0[b] = ceil_div(a.m0[b], AT0);
      a.tiles[b] = a.tiles0[b] * ceil_div(a.m1[b], AT1);
      maxt = std::max(maxt, a.tiles[b]);
      a.in_off[b] = j > 1 ? p.apx_off[b][j - 1] : 0;
      a.a_off[b] = j == p.J ? p.offA[b] : p.apx_off[b][j];
      a.h_off[b] = p.offH[b][j];
    }
    a.in_stride = (int64_t)p.Ny * p.Nx;
    a.s_stride = p.s;
    a.apx_stride = p.apx_total;
    a.first = j == 1;
    a.last = j == p.J;
    a.in_scale = j == 1 ? 1.f / 3.f : 1.f;
    dim3 grid(maxt, kSaraWavelets, np);
    analysis_kernel<<<grid, 256, 0, s>>>(a, x, coef, apx);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
}

bool sara_fused_supported(int lg) { return lg >= 1 && lg <= 32; }

void sara_analysis_prox(const SaraPlan& p, const float* xhat, float* v1, float* apx, const float* weights,
                        const double* beta, int n_groups, int lg, double* l21_acc, cudaStream_t s) {
  upload_filters();
  FHS_CHECK(sara_fused_supported(lg), FHS_ERR_UNSUPPORTED, "fused SARA prox supports at most 32 channels per group");
  for (int j = 1; j <= p.J; ++j) {
    LevelArgs a{};
    int maxt = 0;
    for (int b = 0; b < kSaraWavelets; ++b) {
      a.n0[b] = p.n0[b][j - 1];
      a.n1[b] = p.n1[b][j - 1];
      a.m0[b] = p.n0[b][j];
      a.m1[b] = p.n1[b][j];
      a.tiles0[b] = ceil_div(a.m0[b], AT0);
      a.tiles[b] = a.tiles0[b] * ceil_div(a.m1[b], AT1);
      maxt = std::max(maxt, a.tiles[b]);
      a.in_off[b] = j > 1 ? p.apx_off[b][j - 1] : 0;
      a.a_off[b] = j == p.J ? p.offA[b] : p.apx_off[b][j];
      a.h_off[b] = p.offH[b][j];
    }
    a.in_stride = (int64_t)p.Ny * p.Nx;
    a.s_stride = p.s;
    a.apx_stride = p.apx_total;
    a.first = j == 1;
    a.last = j == p.J;
    a.in_scale = j == 1 ? 1.f / 3.f : 1.f;
    a.dirac = (j == 1 && lg <= kApChunk) ? 1 : 0;   // the split kernel's db1 tiles take the Dirac rows
    a.dirac_off = p.boff[kSaraWavelets];
    dim3 grid(ceil_div(maxt, kApBand) * kSaraWavelets * kApBand, n_groups);
#define FHS_AP(MAXL) launch_analysis_prox<MAXL>(grid, s, a, xhat, apx, v1, weights, beta, lg, l21_acc)
    if (lg <= 1)
      launch_analysis_prox_split<1>(grid, s, a, xhat, apx, v1, weights, beta, lg, l21_acc);
    else if (lg <= 4)
      launch_analysis_prox_split<4>(grid, s, a, xhat, apx, v1, weights, beta, lg, l21_acc);
    else if (lg <= 8)
      launch_analysis_prox_split<8>(grid, s, a, xhat, apx, v1, weights, beta, lg, l21_acc);
    else if (lg <= 16)
      launch_analysis_prox_split<16>(grid, s, a, xhat, apx, v1, weights, beta, lg, l21_acc);
    else
      FHS_AP(32);
#undef FHS_AP
    count_launch();
    FHS_LAUNCH_CHECK();
  }
  if (lg <= kApChunk) return;   // the Dirac rows went with level 1's db1 tiles
  // Dirac part: coefficients are xhat/3
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  const int64_t off = p.boff[kSaraWavelets];
  dim3 grid(nblk(npix), n_groups);
#define FHS_DP(MAXL)                                                                                            \
  l21_prox_kernel<MAXL, true><<<grid, 256, 0, s>>>(v1, nullptr, xhat, weights, beta, p.s, off, npix, lg, nullptr, off, \
                                             l21_acc)
  if (lg <= 1)
    FHS_DP(1);
  else if (lg <= 4)
    FHS_DP(4);
  else if (lg <= 8)
    FHS_DP(8);
  else if (lg <= 16)
    FHS_DP(16);
  else
    FHS_DP(32);
#undef FHS_DP
  count_launch();
  FHS_LAUNCH_CHECK();
}

void sara_dirac(const SaraPlan& p, const float* x, float* coef, int np, cudaStream_t s) {
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  dirac_kernel<<<dim3(nblk(npix), np), 256, 0, s>>>(x, coef, p.s, p.boff[kSaraWavelets], npix);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void sara_synthesis(const SaraPlan& p, const float* coef, float* out, float* apx, int np, float alpha,
                    cudaStream_t s) {
  upload_filters();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(synthesis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(SynSmem)));
    attr[dev] = true;
  }
  for (int j = p.J; j >= 1; --j) {
    SynArgs a{};
    int maxt = 0;
    for (int b = 0; b < kSaraWavelets; ++b) {
      a.m0[b] = p.n0[b][j];
      a.m1[b] = p.n1[b][j];
      a.n0[b] = p.n0[b][j - 1];
      a.n1[b] = p.n1[b][j - 1];
      a.tiles0[b] = ceil_div(a.n0[b], SY);
      a.tiles[b] = a.tiles0[b] * ceil_div(a.n1[b], SX);
      maxt = std::max(maxt, a.tiles[b]);
      a.a_off[b] = j == p.J ? p.offA[b] : p.apx_off[b][j];
      a.h_off[b] = p.offH[b][j];
      a.out_off[b] = j > 1 ? p.apx_off[b][j - 1] : 0;
    }
    a.s_stride = p.s;
    a.apx_stride = p.apx_total;
    a.out_stride = (int64_t)p.Ny * p.Nx;
    a.a_from_coef = j == p.J;
    a.final_level = j == 1;
    a.dirac_off = p.boff[kSaraWavelets];
    a.alpha = alpha / 3.f;
    dim3 grid(a.final_level ? a.tiles[0] : maxt, a.final_level ? 1 : kSaraWavelets, np);
    synthesis_kernel<<<grid, 256, sizeof(SynSmem), s>>>(a, coef, apx, out);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
}

void sara_l21_prox(const SaraPlan& p, float* v1, const float* coef, const float* xhat, const float* weights,
                   const double* beta, int n_groups, int lg, double* l21_partials, cudaStream_t s) {
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  dim3 grid(nblk(p.s), n_groups);
  const int64_t off = p.boff[kSaraWavelets];
#define FHS_L21(MAXL)                                                                                       \
  l21_prox_kernel<MAXL, false><<<grid, 256, 0, s>>>(v1, coef, xhat, weights, beta, p.s, off, npix, lg, l21_partials, 0, \
                                             nullptr)
  if (lg <= 1)
    FHS_L21(1);
  else if (lg <= 4)
    FHS_L21(4);
  else if (lg <= 8)
    FHS_L21(8);
  else if (lg <= 16)
    FHS_L21(16);
  else if (lg <= 32)
    FHS_L21(32);
  else if (lg <= 64)
    FHS_L21(64);
  else
    throw Error(FHS_ERR_UNSUPPORTED, "more than 64 channels per spectral group");
#undef FHS_L21
  count_launch();
  FHS_LAUNCH_CHECK();
}

void sara_row_norms(const SaraPlan& p, const float* coef, const float* x, int n_groups, int lg, float* out,
                    cudaStream_t s) {
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  row_norms_kernel<<<dim3(nblk(p.s), n_groups), 256, 0, s>>>(coef, x, p.s, p.boff[kSaraWavelets], npix, lg,
                                                              out);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
