// Hand-written zero-padded 2-D FFTs of the measurement operator (sm_100a).
//
// A of the reference (apply_scaled_fourier_transform.m:21-24: scale, zero-pad
// to (Ky, Kx) = (oy Ny, ox Nx), FFT2) and the real part of its adjoint, for
// the solvers' real images, with power-of-two grid sides 64..4096:
//
//  forward, image x[L][Nx][Ny] (y fastest) -> half spectrum [L][Kx][Ky/2+1]
//   F1 (along y): each line packs a pair of image columns as the real and
//      imaginary parts of one complex line (zero rows never read: the image
//      occupies Ny of the Ky rows), transforms it and unpacks the two half
//      spectra into their grid columns; the Kx - Nx all-zero columns are
//      never written.
//   F2 (along x, in place): one CTA per group of 4 rows k0 reads the Nx
//      non-zero columns only and writes all Kx.
//  adjoint, full spectrum B[L][Kx][Ky] -> Re(At B) on the image [L][Nx][Ny]
//   I1 (along x): rows k0 <= Ky/2 of the Hermitian part (B(k) + conj
//      B(-k)) / 2, inverse transformed, only the Nx image columns kept
//      (intermediate [L][Nx][Ky/2+1]).
//   I2 (along y, complex-to-real): each line extends a pair of half columns
//      by Hermitian symmetry, inverse transforms them packed as one complex
//      line and keeps the Ny image rows.
//
// Each line is a mixed-radix Stockham FFT (radix 8, then 4 or 2) whose
// length is a compile-time constant.  The first stage takes its 8 inputs per
// thread straight from global memory into registers (no staging pass); the
// other stages exchange through shared memory with a 1-in-8 padded layout
// (conflict-free strided stores).  A butterfly reads one twiddle w from an
// FP64-derived table and forms w^2..w^7 by products.  The lines of a CTA are
// interleaved across neighbouring threads (in the strided passes four
// threads read one 32-byte row segment) with line starts placed so that
// every shared-memory pass is free of bank conflicts.  FP32 arithmetic,
// unnormalised (the adjoint of the forward transform), as the reference's
// fft2 / its adjoint.
#include "measop.cuh"

#include <cmath>
#include <type_traits>

namespace fhs {

namespace {

constexpr int kFftLines = 4;   // lines per CTA of the strided passes (32-byte row segments)

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
__device__ __forceinline__ void dft8(float2* v) {
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

template <bool INV, int R>
__device__ __forceinline__ void butterfly(float2* v) {
  if constexpr (R == 8) {
    dft8<INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else {
    dft2<INV>(v[0], v[1]);
  }
}

// v[r] *= w^r for r = 1..R-1 (w^2.. by products of the table value w)
template <int R>
__device__ __forceinline__ void apply_twiddles(float2* v, float2 w1) {
  if constexpr (R == 2) {
    v[1] = cmulf(v[1], w1);
  } else {
    const float2 w2 = cmulf(w1, w1);
    v[1] = cmulf(v[1], w1);
    v[2] = cmulf(v[2], w2);
    v[3] = cmulf(v[3], cmulf(w2, w1));
    if constexpr (R == 8) {
      const float2 w4 = cmulf(w2, w2);
      v[4] = cmulf(v[4], w4);
      v[5] = cmulf(v[5], cmulf(w4, w1));
      v[6] = cmulf(v[6], cmulf(w4, w2));
      v[7] = cmulf(v[7], cmulf(w4, cmulf(w2, w1)));
    }
  }
}

// One radix-R stage (Ns >= 8) of the Stockham FFT of a line of N values at
// buf[fpad(i)]: butterfly j (of N / R) reads buf[j + r N / R] times
// exp(-+2 pi i r (j mod Ns) / (Ns R)) and writes its radix-R DFT to
// buf[(j / Ns) Ns R + j mod Ns + r Ns].  The TL = N / (8 GM) threads of the
// line own GM groups of 8 values (8 / R butterflies each); all loads finish
// before any store (CTA barrier), so the stage runs in place.
template <bool INV, int N, int NS, int GM>
__device__ __forceinline__ void fft_stage(float2* buf, const float2* __restrict__ tw, int tl) {
  constexpr int R = (N / NS >= 8) ? 8 : N / NS;
  constexpr int NQ = 8 / R, STRIDE = N / R, TWS = N / (NS * R), TL = N / (8 * GM);
  constexpr int PSTRIDE = STRIDE + STRIDE / 8, PNS = NS + NS / 8;   // padded offsets (multiples of 8)
  float2 v[GM][8];
#pragma unroll
  for (int g = 0; g < GM; ++g) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int j = tl + g * TL + q * (N / 8);
      const int k = j & (NS - 1);
      const int base = fpad(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[g][q * R + r] = buf[base + r * PSTRIDE];
      float2 w = __ldg(tw + k * TWS);
      if (INV) w.y = -w.y;
      apply_twiddles<R>(&v[g][q * R], w);
      butterfly<INV, R>(&v[g][q * R]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int g = 0; g < GM; ++g) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int j = tl + g * TL + q * (N / 8);
      const int k = j & (NS - 1);
      const int base = fpad((j - k) * R + k);
#pragma unroll
      for (int r = 0; r < R; ++r) buf[base + r * PNS] = v[g][q * R + r];
    }
  }
  __syncthreads();
}

template <bool INV, int N, int NS, int GM>
__device__ __forceinline__ void fft_stages(float2* buf, const float2* __restrict__ tw, int tl) {
  if constexpr (NS < N) {
    constexpr int R = (N / NS >= 8) ? 8 : N / NS;
    fft_stage<INV, N, NS, GM>(buf, tw, tl);
    fft_stages<INV, N, NS * R, GM>(buf, tw, tl);
  }
}

// FFT of one line of N = 2^m (64 <= N <= 4096) values, element i given by
// load(i), result left at buf[fpad(i)].  The first radix-8 stage (Ns = 1, no
// twiddles) takes its inputs i = j + r N / 8 straight from load(); every
// thread of the CTA calls it (the stages contain CTA barriers).
template <bool INV, int N, int GM, class Load>
__device__ __forceinline__ void line_fft(float2* buf, const float2* __restrict__ tw, int tl, Load load) {
  constexpr int TL = N / (8 * GM);
  float2 v[GM][8];
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    const int j = tl + g * TL;
#pragma unroll
    for (int r = 0; r < 8; ++r) v[g][r] = load(j + r * (N / 8));
  }
#pragma unroll
  for (int g = 0; g < GM; ++g) {
    const int j = tl + g * TL;
    dft8<INV>(v[g]);
#pragma unroll
    for (int r = 0; r < 8; ++r) buf[9 * j + r] = v[g][r];   // fpad(8 j + r)
  }
  __syncthreads();
  fft_stages<INV, N, 8, GM>(buf, tw, tl);
}

// image row iy of grid row ky (-1: a padding row)
__device__ __forceinline__ int image_index(int k, int n, int K) {
  const int h = n >> 1;
  return k < h ? k + h : (k >= K - h ? k - K + h : -1);
}

// Shared-memory layout of the LPC lines of a CTA.  Lines are interleaved
// across threads (thread t: line t mod LPC, butterfly index t / LPC), so a
// half-warp -- the unit of a 64-bit shared access -- holds 16 / LPC
// consecutive elements of each of its LPC lines, which lie inside one padding
// group of 8.  Line starts 16 / LPC slots (of 8 bytes) apart modulo 16 give
// each line of the half-warp its own banks: one wavefront per half-warp for
// the consecutive reads and writes of every stage and for the first stage's
// stores at 9 j + r.
constexpr int line_len(int N, int LPC) {
  return N + N / 8 + ((16 / LPC - (N + N / 8) % 16) % 16 + 16) % 16;
}

// F1: x[L][Nx][Ny] (scaled by sy, sx) -> columns of the half spectrum; LPC
// lines (column pairs) per CTA, TL threads each
template <int LOGN, int GM, int LPC>
__global__ void __launch_bounds__((1 << LOGN) / (8 * GM) * LPC) fft_f1_kernel(
    const float* __restrict__ x, const float* __restrict__ sy, const float* __restrict__ sx,
    const float2* __restrict__ tw, int Ny, int Nx, int Kx, int p0, float2* __restrict__ half) {
  constexpr int N = 1 << LOGN, TL = N / (8 * GM), Kh = N / 2 + 1;
  extern __shared__ float2 f1_sm[];
  const int line = threadIdx.x % LPC, tl = threadIdx.x / LPC;
  float2* buf = f1_sm + line * line_len(N, LPC);
  const int pair = blockIdx.x * LPC + line;
  const bool active = pair < Nx / 2;
  const int ia = 2 * (active ? pair : 0), ib = ia + 1;
  const float* xa = x + ((size_t)blockIdx.y * Nx + ia) * Ny;
  const float* xb = xa + Ny;
  const float sxa = __ldg(sx + ia), sxb = __ldg(sx + ib);
  line_fft<false, N, GM>(buf, tw, tl, [&](int k) {
    const int iy = image_index(k, Ny, N);
    if (!active || iy < 0) return make_float2(0.f, 0.f);
    const float s = __ldg(sy + iy);
    return make_float2(__ldg(xa + iy) * s * sxa, __ldg(xb + iy) * s * sxb);
  });
  if (!active) return;
  const int plane = p0 + blockIdx.y;
  const int kxa = ia - Nx / 2 + (ia < Nx / 2 ? Kx : 0), kxb = ib - Nx / 2 + (ib < Nx / 2 ? Kx : 0);
  float2* ca = half + ((size_t)plane * Kx + kxa) * Kh;
  float2* cb = half + ((size_t)plane * Kx + kxb) * Kh;
  for (int k = tl; k < Kh; k += TL) {
    const float2 z = buf[fpad(k)];
    const float2 zm = buf[fpad((N - k) & (N - 1))];
    // A = (Z + conj Zm) / 2, B = (Z - conj Zm) / (2i)
    ca[k] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    cb[k] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
  }
}

// F2: along x (N = Kx), rows k0 .. k0 + 3 of the half spectrum, in place
template <int LOGN, int GM>
__global__ void __launch_bounds__((1 << LOGN) / (8 * GM) * kFftLines, GM <= 2 ? 2 : 1) fft_f2_kernel(
    const float2* __restrict__ tw, int Nx, int Ky, int p0, float2* __restrict__ half) {
  constexpr int N = 1 << LOGN, TL = N / (8 * GM);
  extern __shared__ float2 f2_sm[];
  const int b = threadIdx.x & (kFftLines - 1), tl = threadIdx.x / kFftLines;
  float2* buf = f2_sm + b * line_len(N, kFftLines);
  const int Kh = Ky / 2 + 1;
  const int row = blockIdx.x * kFftLines + b;
  const bool valid = row < Kh;
  float2* hp = half + (size_t)(p0 + blockIdx.y) * N * Kh + (valid ? row : 0);
  line_fft<false, N, GM>(buf, tw, tl, [&](int kx) {
    if (!valid || (kx >= Nx / 2 && kx < N - Nx / 2)) return make_float2(0.f, 0.f);
    return hp[(size_t)kx * Kh];
  });
  if (!valid) return;
  for (int kx = tl; kx < N; kx += TL) hp[(size_t)kx * Kh] = buf[fpad(kx)];
}

// I1: rows k0 .. k0 + 3 (<= Ky/2) of the Hermitian part of B, inverse along
// x (N = Kx), the Nx image columns kept: U[L][Nx][Kh]
template <int LOGN, int GM>
__global__ void __launch_bounds__((1 << LOGN) / (8 * GM) * kFftLines, GM <= 2 ? 2 : 1) fft_i1_kernel(
    const float2* __restrict__ tw, const float2* __restrict__ B, int Nx, int Ky, int p0, float2* __restrict__ U) {
  constexpr int N = 1 << LOGN, TL = N / (8 * GM);
  extern __shared__ float2 i1_sm[];
  const int b = threadIdx.x & (kFftLines - 1), tl = threadIdx.x / kFftLines;
  float2* buf = i1_sm + b * line_len(N, kFftLines);
  const int Kh = Ky / 2 + 1;
  const int plane = p0 + blockIdx.y;
  const int ky0 = blockIdx.x * kFftLines + b;
  const bool valid = ky0 < Kh;
  const int ky = valid ? ky0 : 0;
  const int mky = (Ky - ky) & (Ky - 1);
  const float2* bp = B + (size_t)plane * N * Ky;
  line_fft<true, N, GM>(buf, tw, tl, [&](int kx) {
    if (!valid) return make_float2(0.f, 0.f);
    const float2 a = bp[(size_t)kx * Ky + ky];
    const float2 m = bp[(size_t)((N - kx) & (N - 1)) * Ky + mky];
    return make_float2(0.5f * (a.x + m.x), 0.5f * (a.y - m.y));   // Hermitian part
  });
  if (!valid) return;
  float2* up = U + (size_t)plane * Nx * Kh + ky;
  for (int ix = tl; ix < Nx; ix += TL) {
    const int kx = ix - Nx / 2 + (ix < Nx / 2 ? N : 0);
    up[(size_t)ix * Kh] = buf[fpad(kx)];
  }
}

// I2: columns ia, ib of U, complex-to-real inverse along y (N = Ky), the Ny
// image rows kept: out[L][Nx][Ny] = Re(At B) without the scaling factors
template <int LOGN, int GM, int LPC>
__global__ void __launch_bounds__((1 << LOGN) / (8 * GM) * LPC) fft_i2_kernel(
    const float2* __restrict__ tw, const float2* __restrict__ U, int Ny, int Nx, int p0, float* __restrict__ out) {
  constexpr int N = 1 << LOGN, TL = N / (8 * GM), Kh = N / 2 + 1;
  extern __shared__ float2 i2_sm[];
  const int line = threadIdx.x % LPC, tl = threadIdx.x / LPC;
  float2* buf = i2_sm + line * line_len(N, LPC);
  const int pair = blockIdx.x * LPC + line;
  const bool active = pair < Nx / 2;
  const int ia = 2 * (active ? pair : 0), ib = ia + 1;
  const float2* ua = U + ((size_t)(p0 + blockIdx.y) * Nx + ia) * Kh;
  const float2* ub = ua + Kh;
  line_fft<true, N, GM>(buf, tw, tl, [&](int k) {
    if (!active) return make_float2(0.f, 0.f);
    const bool hi = k >= Kh;   // Hermitian extension
    const int kk = hi ? N - k : k;
    float2 a = ua[kk], c = ub[kk];
    if (hi) {
      a.y = -a.y;
      c.y = -c.y;
    }
    return make_float2(a.x - c.y, a.y + c.x);   // a + i c
  });
  if (!active) return;
  float* oa = out + ((size_t)blockIdx.y * Nx + ia) * Ny;
  float* ob = oa + Ny;
  for (int iy = tl; iy < Ny; iy += TL) {
    const int k = iy - Ny / 2 + (iy < Ny / 2 ? N : 0);
    const float2 z = buf[fpad(k)];
    oa[iy] = z.x;
    ob[iy] = z.y;
  }
}

bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

int log2i(int n) {
  int m = 0;
  while ((1 << m) < n) ++m;
  return m;
}

// launch shapes: contiguous passes (F1, I2) use TL = min(N / 8, 256) threads
// per line and LPC >= 2 lines per CTA (at least 128 threads); strided passes
// (F2, I1) use 4 lines of TL = min(N / 8, 128) threads
template <int LOGN>
struct Shape {
  static constexpr int N = 1 << LOGN;
  static constexpr int GMc = N > 2048 ? 2 : 1;
  static constexpr int TLc = N / (8 * GMc);
  static constexpr int LPC = TLc >= 64 ? 2 : 128 / TLc;
  static constexpr int GMs = N > 1024 ? N / 1024 : 1;
  static constexpr int TLs = N / (8 * GMs);
  static constexpr size_t smem_c = (size_t)LPC * line_len(N, LPC) * sizeof(float2);
  static constexpr size_t smem_s = (size_t)kFftLines * line_len(N, kFftLines) * sizeof(float2);
};

template <int LOGN>
void set_attributes() {
  using S = Shape<LOGN>;
  FHS_CUDA(cudaFuncSetAttribute(fft_f1_kernel<LOGN, S::GMc, S::LPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)S::smem_c));
  FHS_CUDA(cudaFuncSetAttribute(fft_i2_kernel<LOGN, S::GMc, S::LPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)S::smem_c));
  FHS_CUDA(cudaFuncSetAttribute(fft_f2_kernel<LOGN, S::GMs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)S::smem_s));
  FHS_CUDA(cudaFuncSetAttribute(fft_i1_kernel<LOGN, S::GMs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)S::smem_s));
}

template <int LOGN>
void launch_f1(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s) {
  using S = Shape<LOGN>;
  const dim3 grid((op->Nx / 2 + S::LPC - 1) / S::LPC, np);
  fft_f1_kernel<LOGN, S::GMc, S::LPC><<<grid, S::TLc * S::LPC, S::smem_c, s>>>(
      x, op->sy.p, op->sx.p, op->tw_y.p, op->Ny, op->Nx, op->Kx, p0, op->gridA.p);
}

template <int LOGN>
void launch_f2(const MeasOp* op, int p0, int np, cudaStream_t s) {
  using S = Shape<LOGN>;
  const int Kh = op->Ky / 2 + 1;
  const dim3 grid((Kh + kFftLines - 1) / kFftLines, np);
  fft_f2_kernel<LOGN, S::GMs><<<grid, S::TLs * kFftLines, S::smem_s, s>>>(op->tw_x.p, op->Nx, op->Ky, p0,
                                                                         op->gridA.p);
}

template <int LOGN>
void launch_i1(const MeasOp* op, int p0, int np, cudaStream_t s) {
  using S = Shape<LOGN>;
  const int Kh = op->Ky / 2 + 1;
  const dim3 grid((Kh + kFftLines - 1) / kFftLines, np);
  fft_i1_kernel<LOGN, S::GMs><<<grid, S::TLs * kFftLines, S::smem_s, s>>>(op->tw_x.p, op->gridB.p, op->Nx,
                                                                         op->Ky, p0, op->gridA.p);
}

template <int LOGN>
void launch_i2(const MeasOp* op, float* out, int p0, int np, cudaStream_t s) {
  using S = Shape<LOGN>;
  const dim3 grid((op->Nx / 2 + S::LPC - 1) / S::LPC, np);
  fft_i2_kernel<LOGN, S::GMc, S::LPC><<<grid, S::TLc * S::LPC, S::smem_c, s>>>(
      op->tw_y.p, op->gridA.p, op->Ny, op->Nx, p0, out);
}

// f(integral_constant<LOGN>) for the runtime side n (a power of two in 64..4096)
template <class F>
void by_size(int n, F&& f) {
  switch (log2i(n)) {
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 10: f(std::integral_constant<int, 10>{}); break;
    case 11: f(std::integral_constant<int, 11>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    default: FHS_CHECK(false, FHS_ERR_UNSUPPORTED, "FFT side must be a power of two in 64..4096");
  }
}

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
    for (int m = 6; m <= 12; ++m) by_size(1 << m, [](auto lg) { set_attributes<decltype(lg)::value>(); });
    attr[dev] = true;
  }
}

void fft_forward_half(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s) {
  by_size(op->Ky, [&](auto lg) { launch_f1<decltype(lg)::value>(op, x, p0, np, s); });
  count_launch();
  FHS_LAUNCH_CHECK();
  by_size(op->Kx, [&](auto lg) { launch_f2<decltype(lg)::value>(op, p0, np, s); });
  count_launch();
  FHS_LAUNCH_CHECK();
}

void fft_inverse_real(const MeasOp* op, float* out, int p0, int np, cudaStream_t s) {
  by_size(op->Kx, [&](auto lg) { launch_i1<decltype(lg)::value>(op, p0, np, s); });
  count_launch();
  FHS_LAUNCH_CHECK();
  by_size(op->Ky, [&](auto lg) { launch_i2<decltype(lg)::value>(op, out, p0, np, s); });
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
