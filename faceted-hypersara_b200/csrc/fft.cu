// Hand-written zero-padded 2-D FFTs of the measurement operator (sm_100a).
//
// A of the reference (apply_scaled_fourier_transform.m:21-24: scale, zero-pad
// to (Ky, Kx) = (oy Ny, ox Nx), FFT2) and the real part of its adjoint, for
// the solvers' real images, with power-of-two grid sides 64..4096:
//
//  forward, image x[L][Nx][Ny] (y fastest) -> half spectrum [L][Kx][Ky/2+1]
//   F1 (along y): one CTA per pair of image columns packs them as the real
//      and imaginary parts of one complex line (zero rows never read: the
//      image occupies Ny of the Ky rows), transforms it and unpacks the two
//      half spectra into their grid columns; the Kx - Nx all-zero columns are
//      never written.
//   F2 (along x, in place): one CTA per group of 4 rows k0 reads the Nx
//      non-zero columns only and writes all Kx.
//  adjoint, full spectrum B[L][Kx][Ky] -> Re(At B) on the image [L][Nx][Ny]
//   I1 (along x): rows k0 <= Ky/2 of the Hermitian part (B(k) + conj
//      B(-k)) / 2, inverse transformed, only the Nx image columns kept
//      (intermediate [L][Nx][Ky/2+1]).
//   I2 (along y, complex-to-real): one CTA per pair of image columns extends
//      the two half lines by Hermitian symmetry, inverse transforms them
//      packed as one complex line and keeps the Ny image rows.
// Each line is a mixed-radix Stockham FFT (radix 8, then 4 or 2) in shared
// memory with a 1-in-8 padded layout (conflict-free strided stores) and an
// FP64-derived twiddle table; FP32 arithmetic, unnormalised (the adjoint of
// the forward transform), as the reference's fft2 / its adjoint.
#include "measop.cuh"

#include <cmath>

namespace fhs {

namespace {

constexpr int kFftLines = 4;   // lines per CTA of the strided passes (32-byte row segments)
constexpr int kLoadUnroll = 8; // global loads in flight per thread while a line is staged

__device__ __forceinline__ int fpad(int a) { return a + (a >> 3); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by sign * i (INV: +i, forward: -i)
template <bool INV>
__device__ __forceinline__ float2 mul_i(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  const float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  const float2 e0 = cadd(a0, a2), e1 = csub(a0, a2);
  const float2 o0 = cadd(a1, a3), o1 = mul_i<INV>(csub(a1, a3));
  a0 = cadd(e0, o0);
  a2 = csub(e0, o0);
  a1 = cadd(e1, o1);
  a3 = csub(e1, o1);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  const float h = 0.70710678118654752f;
  // w8^k = exp(sign i pi k / 4)
  const float2 w1 = INV ? make_float2(h, h) : make_float2(h, -h);
  const float2 w3 = INV ? make_float2(-h, h) : make_float2(-h, -h);
  o1 = cmulf(o1, w1);
  o2 = mul_i<INV>(o2);
  o3 = cmulf(o3, w3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// One radix-R stage of the Stockham FFT of a line: butterfly j (of N / R)
// reads buf[j + r N / R] times exp(-+2 pi i r (j mod Ns) / (Ns R)) and
// writes the radix-R DFT to buf[(j / Ns) Ns R + j mod Ns + r Ns].  A thread
// owns G <= 2 groups of 8 values (8 / R butterflies each); all loads finish
// before any store (CTA barrier), so the stage runs in place.
template <bool INV, int R, int GM>
__device__ __forceinline__ void fft_stage(float2* buf, const float2* __restrict__ tw, int N, int Ns, int tl, int TL) {
  constexpr int NQ = 8 / R;
  const int stride = N / R, tws = N / (Ns * R);
  float2 v[GM][8];
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    {
      const int j0 = tl + g * TL;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int j = j0 + q * (N >> 3);
        const int k = j & (Ns - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          float2 x = buf[fpad(j + r * stride)];
          if (r > 0 && k > 0) {
            float2 w = __ldg(tw + r * k * tws);
            if (INV) w.y = -w.y;
            x = cmulf(x, w);
          }
          v[g][q * R + r] = x;
        }
      }
      if (R == 8) {
        dft8<INV>(v[g]);
      } else if (R == 4) {
        dft4<INV>(v[g][0], v[g][1], v[g][2], v[g][3]);
        dft4<INV>(v[g][4], v[g][5], v[g][6], v[g][7]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) dft2<INV>(v[g][2 * q], v[g][2 * q + 1]);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    {
      const int j0 = tl + g * TL;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int j = j0 + q * (N >> 3);
        const int k = j & (Ns - 1);
        const int d = (j - k) * R + k;   // (j / Ns) Ns R + j mod Ns
#pragma unroll
        for (int r = 0; r < R; ++r) buf[fpad(d + r * Ns)] = v[g][q * R + r];
      }
    }
  }
  __syncthreads();
}

// In-place FFT of one line of N = 2^m (64 <= N <= 4096) complex values held
// at buf[fpad(i)], by the TL threads tl = 0..TL-1 of this line, TL = N / (8 GM).
// tw[k] = exp(-2 pi i k / N).  Every thread of the CTA calls it (the stages
// contain CTA barriers).  Radix 8 while N / Ns >= 8, then 4 or 2.
template <bool INV, int GM>
__device__ void line_fft(float2* buf, const float2* __restrict__ tw, int N, int tl, int TL) {
  for (int Ns = 1; Ns < N;) {
    const int R = (N / Ns >= 8) ? 8 : N / Ns;
    if (R == 8)
      fft_stage<INV, 8, GM>(buf, tw, N, Ns, tl, TL);
    else if (R == 4)
      fft_stage<INV, 4, GM>(buf, tw, N, Ns, tl, TL);
    else
      fft_stage<INV, 2, GM>(buf, tw, N, Ns, tl, TL);
    Ns *= R;
  }
}

// image row iy of grid row ky (-1: a padding row)
__device__ __forceinline__ int image_index(int k, int n, int K) {
  const int h = n >> 1;
  return k < h ? k + h : (k >= K - h ? k - K + h : -1);
}

// F1: x[L][Nx][Ny] (scaled by sy, sx) -> columns of the half spectrum
template <int GM>
__global__ void __launch_bounds__(256) fft_f1_kernel(const float* __restrict__ x, const float* __restrict__ sy,
                                                     const float* __restrict__ sx, const float2* __restrict__ tw,
                                                     int Ny, int Nx, int Ky, int Kx, int p0,
                                                     float2* __restrict__ half) {
  extern __shared__ float2 f1_sm[];
  float2* buf = f1_sm;
  const int plane = p0 + blockIdx.y;
  const int ia = 2 * blockIdx.x, ib = ia + 1;
  const int Kh = Ky / 2 + 1;
  const float* xa = x + ((size_t)blockIdx.y * Nx + ia) * Ny;
  const float* xb = xa + Ny;
  const float sxa = sx[ia], sxb = sx[ib];
  for (int k0 = 0; k0 < Ky; k0 += kLoadUnroll * blockDim.x) {
    float2 v[kLoadUnroll];
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int k = k0 + u * blockDim.x + threadIdx.x;
      const int iy = k < Ky ? image_index(k, Ny, Ky) : -1;
      v[u] = make_float2(0.f, 0.f);
      if (iy >= 0) v[u] = make_float2(xa[iy] * sy[iy] * sxa, xb[iy] * sy[iy] * sxb);
    }
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int k = k0 + u * blockDim.x + threadIdx.x;
      if (k < Ky) buf[fpad(k)] = v[u];
    }
  }
  __syncthreads();
  line_fft<false, GM>(buf, tw, Ky, threadIdx.x, blockDim.x);
  const int kxa = ia - Nx / 2 + (ia < Nx / 2 ? Kx : 0), kxb = ib - Nx / 2 + (ib < Nx / 2 ? Kx : 0);
  float2* ca = half + ((size_t)plane * Kx + kxa) * Kh;
  float2* cb = half + ((size_t)plane * Kx + kxb) * Kh;
  for (int k = threadIdx.x; k < Kh; k += blockDim.x) {
    const float2 z = buf[fpad(k)];
    const float2 zm = buf[fpad(k == 0 ? 0 : Ky - k)];
    // A = (Z + conj Zm) / 2, B = (Z - conj Zm) / (2i)
    ca[k] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    cb[k] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
  }
}

// F2: along x, rows k0 .. k0 + 3 of the half spectrum, in place
template <int GM>
__global__ void __launch_bounds__(512, 2) fft_f2_kernel(const float2* __restrict__ tw, int Nx, int Ky, int Kx, int p0,
                                                      float2* __restrict__ half) {
  extern __shared__ float2 f2_sm[];
  float2* buf = f2_sm;
  const int Kh = Ky / 2 + 1;
  const int plane = p0 + blockIdx.y;
  const int k0 = blockIdx.x * kFftLines;
  const int nl = min(kFftLines, Kh - k0);
  const int lp = Kx + (Kx >> 3);   // padded line length
  float2* hp = half + (size_t)plane * Kx * Kh;
  // 8 independent loads in flight per thread, then the shared-memory stores
  for (int t0 = 0; t0 < Kx * kFftLines; t0 += kLoadUnroll * blockDim.x) {
    float2 v[kLoadUnroll];
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int t = t0 + u * blockDim.x + threadIdx.x;
      const int kx = t / kFftLines, b = t - kx * kFftLines;
      v[u] = make_float2(0.f, 0.f);
      if (t < Kx * kFftLines && b < nl && (kx < Nx / 2 || kx >= Kx - Nx / 2)) v[u] = hp[(size_t)kx * Kh + k0 + b];
    }
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int t = t0 + u * blockDim.x + threadIdx.x;
      const int kx = t / kFftLines, b = t - kx * kFftLines;
      if (t < Kx * kFftLines) buf[b * lp + fpad(kx)] = v[u];
    }
  }
  __syncthreads();
  const int TL = blockDim.x / kFftLines;
  line_fft<false, GM>(buf + (threadIdx.x / TL) * lp, tw, Kx, threadIdx.x % TL, TL);
  for (int t = threadIdx.x; t < Kx * kFftLines; t += blockDim.x) {
    const int kx = t / kFftLines, b = t - kx * kFftLines;
    if (b < nl) hp[(size_t)kx * Kh + k0 + b] = buf[b * lp + fpad(kx)];
  }
}

// I1: rows k0 .. k0 + 3 (<= Ky/2) of the Hermitian part of B, inverse along
// x, the Nx image columns kept: U[L][Nx][Kh]
template <int GM>
__global__ void __launch_bounds__(512, 2) fft_i1_kernel(const float2* __restrict__ tw, const float2* __restrict__ B,
                                                      int Nx, int Ky, int Kx, int p0, float2* __restrict__ U) {
  extern __shared__ float2 i1_sm[];
  float2* buf = i1_sm;
  const int Kh = Ky / 2 + 1;
  const int plane = p0 + blockIdx.y;
  const int k0 = blockIdx.x * kFftLines;
  const int nl = min(kFftLines, Kh - k0);
  const int lp = Kx + (Kx >> 3);
  const float2* bp = B + (size_t)plane * Kx * Ky;
  for (int t0 = 0; t0 < Kx * kFftLines; t0 += kLoadUnroll * blockDim.x) {
    float2 va[kLoadUnroll], vm[kLoadUnroll];
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int t = t0 + u * blockDim.x + threadIdx.x;
      const int kx = t / kFftLines, b = t - kx * kFftLines;
      va[u] = vm[u] = make_float2(0.f, 0.f);
      if (t < Kx * kFftLines && b < nl) {
        const int ky = k0 + b;
        va[u] = bp[(size_t)kx * Ky + ky];
        vm[u] = bp[(size_t)(kx == 0 ? 0 : Kx - kx) * Ky + (ky == 0 ? 0 : Ky - ky)];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int t = t0 + u * blockDim.x + threadIdx.x;
      const int kx = t / kFftLines, b = t - kx * kFftLines;
      if (t < Kx * kFftLines)   // Hermitian part (B(k) + conj B(-k)) / 2
        buf[b * lp + fpad(kx)] = make_float2(0.5f * (va[u].x + vm[u].x), 0.5f * (va[u].y - vm[u].y));
    }
  }
  __syncthreads();
  const int TL = blockDim.x / kFftLines;
  line_fft<true, GM>(buf + (threadIdx.x / TL) * lp, tw, Kx, threadIdx.x % TL, TL);
  float2* up = U + (size_t)plane * Nx * Kh;
  for (int t = threadIdx.x; t < Nx * kFftLines; t += blockDim.x) {
    const int ix = t / kFftLines, b = t - ix * kFftLines;
    const int kx = ix - Nx / 2 + (ix < Nx / 2 ? Kx : 0);
    if (b < nl) up[(size_t)ix * Kh + k0 + b] = buf[b * lp + fpad(kx)];
  }
}

// I2: columns ia, ib of U, complex-to-real inverse along y, the Ny image
// rows kept: out[L][Nx][Ny] = Re(At B) without the scaling factors
template <int GM>
__global__ void __launch_bounds__(256) fft_i2_kernel(const float2* __restrict__ tw, const float2* __restrict__ U,
                                                     int Ny, int Nx, int Ky, int p0, float* __restrict__ out) {
  extern __shared__ float2 i2_sm[];
  float2* buf = i2_sm;
  const int Kh = Ky / 2 + 1;
  const int plane = p0 + blockIdx.y;
  const int ia = 2 * blockIdx.x, ib = ia + 1;
  const float2* ua = U + ((size_t)plane * Nx + ia) * Kh;
  const float2* ub = ua + Kh;
  for (int k0 = 0; k0 < Ky; k0 += kLoadUnroll * blockDim.x) {
    float2 va[kLoadUnroll], vb[kLoadUnroll];
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int k = k0 + u * blockDim.x + threadIdx.x;
      const int kk = k < Kh ? k : Ky - k;
      va[u] = vb[u] = make_float2(0.f, 0.f);
      if (k < Ky) {
        va[u] = ua[kk];
        vb[u] = ub[kk];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadUnroll; ++u) {
      const int k = k0 + u * blockDim.x + threadIdx.x;
      float2 a = va[u], b = vb[u];
      if (k >= Kh) {   // Hermitian extension
        a.y = -a.y;
        b.y = -b.y;
      }
      if (k < Ky) buf[fpad(k)] = make_float2(a.x - b.y, a.y + b.x);   // a + i b
    }
  }
  __syncthreads();
  line_fft<true, GM>(buf, tw, Ky, threadIdx.x, blockDim.x);
  float* oa = out + ((size_t)blockIdx.y * Nx + ia) * Ny;
  float* ob = oa + Ny;
  for (int iy = threadIdx.x; iy < Ny; iy += blockDim.x) {
    const int k = iy - Ny / 2 + (iy < Ny / 2 ? Ky : 0);
    const float2 z = buf[fpad(k)];
    oa[iy] = z.x;
    ob[iy] = z.y;
  }
}

size_t line_smem(int N, int lines) { return (size_t)lines * (N + N / 8) * sizeof(float2); }

bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

}  // namespace

bool measop_own_fft(const MeasOp* op) {
  return pow2_in(op->Ky, 64, 4096) && pow2_in(op->Kx, 64, 4096) && (op->Nx % 2 == 0);
}

void measop_fft_tables(MeasOp* op, cudaStream_t s) {
  auto table = [&](int N, DevBuf<float2>& t) {
    std::vector<float2> h(N);
    for (int k = 0; k < N; ++k) {
      const double a = -2.0 * M_PI * (double)k / (double)N;
      h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    t.alloc(N);
    t.upload(h.data(), N, s);
  };
  table(op->Ky, op->tw_y);
  table(op->Kx, op->tw_x);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    const int big = (int)line_smem(4096, kFftLines), one = (int)line_smem(4096, 1);
    FHS_CUDA(cudaFuncSetAttribute(fft_f2_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_f2_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_f2_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_i1_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_i1_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_i1_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FHS_CUDA(cudaFuncSetAttribute(fft_f1_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
    FHS_CUDA(cudaFuncSetAttribute(fft_f1_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
    FHS_CUDA(cudaFuncSetAttribute(fft_i2_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
    FHS_CUDA(cudaFuncSetAttribute(fft_i2_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
    attr[dev] = true;
  }
}

// threads per line of the contiguous passes (one group of 8 values per
// thread up to N = 2048, two at 4096) and of the strided passes (4 lines per
// CTA, at most 128 threads per line: two groups per thread at N = 2048)
static int line_threads(int N) { return std::min(256, N / 8); }
static int strided_threads(int N) { return std::min(128, N / 8); }

void fft_forward_half(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s) {
  const int Kh = op->Ky / 2 + 1;
  const dim3 g1(op->Nx / 2, np), g2((Kh + kFftLines - 1) / kFftLines, np);
  const int t1 = line_threads(op->Ky), t2 = kFftLines * strided_threads(op->Kx);
  const size_t s1 = line_smem(op->Ky, 1), s2 = line_smem(op->Kx, kFftLines);
  if (op->Ky > 2048)
    fft_f1_kernel<2><<<g1, t1, s1, s>>>(x, op->sy.p, op->sx.p, op->tw_y.p, op->Ny, op->Nx, op->Ky, op->Kx, p0,
                                        op->gridA.p);
  else
    fft_f1_kernel<1><<<g1, t1, s1, s>>>(x, op->sy.p, op->sx.p, op->tw_y.p, op->Ny, op->Nx, op->Ky, op->Kx, p0,
                                        op->gridA.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  if (op->Kx / 8 / strided_threads(op->Kx) == 4)
    fft_f2_kernel<4><<<g2, t2, s2, s>>>(op->tw_x.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  else if (op->Kx / 8 / strided_threads(op->Kx) == 2)
    fft_f2_kernel<2><<<g2, t2, s2, s>>>(op->tw_x.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  else
    fft_f2_kernel<1><<<g2, t2, s2, s>>>(op->tw_x.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void fft_inverse_real(const MeasOp* op, float* out, int p0, int np, cudaStream_t s) {
  const int Kh = op->Ky / 2 + 1;
  const dim3 g1((Kh + kFftLines - 1) / kFftLines, np), g2(op->Nx / 2, np);
  const int t1 = kFftLines * strided_threads(op->Kx), t2 = line_threads(op->Ky);
  const size_t s1 = line_smem(op->Kx, kFftLines), s2 = line_smem(op->Ky, 1);
  if (op->Kx / 8 / strided_threads(op->Kx) == 4)
    fft_i1_kernel<4><<<g1, t1, s1, s>>>(op->tw_x.p, op->gridB.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  else if (op->Kx / 8 / strided_threads(op->Kx) == 2)
    fft_i1_kernel<2><<<g1, t1, s1, s>>>(op->tw_x.p, op->gridB.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  else
    fft_i1_kernel<1><<<g1, t1, s1, s>>>(op->tw_x.p, op->gridB.p, op->Nx, op->Ky, op->Kx, p0, op->gridA.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  if (op->Ky > 2048)
    fft_i2_kernel<2><<<g2, t2, s2, s>>>(op->tw_y.p, op->gridA.p, op->Ny, op->Nx, op->Ky, p0, out);
  else
    fft_i2_kernel<1><<<g2, t2, s2, s>>>(op->tw_y.p, op->gridA.p, op->Ny, op->Nx, op->Ky, p0, out);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
