// Learned warm start: a BF16 U-Net with hand-written training and inference
// kernels on B200 (sm_100a).
//
// The network maps one normalised dirty image (a channel of the back-projected
// cube) to an initial estimate of the solver's solution; the solvers take it
// as their xinit (src/fhs/facetHyperSARA.m:1-6, varargin{1}, applied at
// :347-350).  It has no counterpart in the reference.
//
// Architecture (4 levels, 32 base channels, 2,140,065 parameters): encoder
// levels of two 3x3 convolutions + ReLU with 32, 64, 128 and 256 channels,
// 2x2 average pooling between them; decoder levels that upsample (nearest,
// 2x), convolve (3x3 + ReLU) to the level's width, concatenate the encoder
// feature map of that level and apply two more 3x3 convolutions + ReLU; a
// 1x1 convolution to one channel.  No residual path to the input: the
// normalised dirty image is about the beam area (tens of pixels) times
// larger than the sky it maps to, so an identity path only has to be
// cancelled first.
//
// Kernels:
//  * conv3x3_kernel: implicit GEMM on the tensor cores (mma.sync m16n8k16,
//    BF16 operands, FP32 accumulation): a CTA computes an 8x8 pixel tile x 64
//    output channels; per 32-channel slice of the input it stages the 10x10
//    input halo (NHWC, fused nearest upsampling and channel concatenation)
//    and the slice of the weights in shared memory (row pitch 40 elements:
//    the 16-byte rows of an ldmatrix fall on distinct bank groups); epilogue
//    bias + ReLU -> BF16.  The data gradient of a layer is the same kernel on
//    the flipped, transposed weights.
//  * wgrad_kernel: weight gradient, a GEMM over pixels per tap
//    (ldmatrix.trans of the pixel-major gradient and input tiles), FP32
//    atomics into the gradient buffer once per CTA.
//  * pooling, upsampling adjoint, ReLU mask, 1x1 head, loss and Adam kernels.
// Activations and activation gradients are BF16 (NHWC), parameters and their
// gradients FP32 (Adam moments FP32), all accumulation FP32.
#include <cuda_bf16.h>

#include <cmath>
#include <memory>
#include <vector>

#include "common.cuh"

namespace fhs {

namespace {

using bf16 = __nv_bfloat16;

constexpr int kCT = 64;      // output channels per conv CTA
constexpr int kCK = 32;      // input channels per staged slice
constexpr int kPitch = 40;   // bf16 per staged row (32 + 8 pad)
constexpr int kHalo = 10;    // 8x8 tile + 1-pixel ring

// A channel slice of an NHWC tensor: element (n, y, x, c) at
// p[((n * H + y) * W + x) * pitch + c].
struct TView {
  const bf16* p;
  int C, pitch;
};

struct ConvArgs {
  TView in0, in1;   // channels [0, in0.C) from in0, [in0.C, in0.C + in1.C) from in1
  int up;           // 1: inputs are (H/2, W/2) maps read through a nearest 2x upsample
  int N, H, W;      // output size
  int Cin, Cpad, Cout;
  const bf16* w;    // [Cout][9][Cpad], tap = 3 * ky + kx (offsets ky - 1, kx - 1)
  const float* bias;
  int relu;
  bf16* out;
  int out_pitch;
};

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

// D += A (16x16, row) * B (16x8, col), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 8 consecutive channels c0..c0+7 of input pixel (n, y, x) of the (possibly
// concatenated, upsampled) conv input; zeros outside the image or past Cin.
__device__ __forceinline__ uint4 load_in8(const ConvArgs& a, int n, int y, int x, int c0) {
  uint4 z = make_uint4(0u, 0u, 0u, 0u);
  if (y < 0 || y >= a.H || x < 0 || x >= a.W || c0 >= a.Cin) return z;
  int h = a.H, w = a.W;
  if (a.up) {
    y >>= 1;
    x >>= 1;
    h >>= 1;
    w >>= 1;
  }
  const size_t pix = ((size_t)n * h + y) * w + x;
  const int C0 = a.in0.C;
  if (c0 + 8 <= C0 && (C0 & 7) == 0 && (a.in0.pitch & 7) == 0)
    return *reinterpret_cast<const uint4*>(a.in0.p + pix * a.in0.pitch + c0);
  if (c0 >= C0 && c0 + 8 <= a.Cin && ((c0 - C0) & 7) == 0 && (a.in1.pitch & 7) == 0)
    return *reinterpret_cast<const uint4*>(a.in1.p + pix * a.in1.pitch + (c0 - C0));
  bf16 v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int c = c0 + k;
    v[k] = c < C0 ? a.in0.p[pix * a.in0.pitch + c]
                  : (c < a.Cin ? a.in1.p[pix * a.in1.pitch + (c - C0)] : __float2bfloat16(0.f));
  }
  return *reinterpret_cast<const uint4*>(v);
}

// 3x3 convolution, stride 1, zero padding 1 (cross-correlation, as the
// usual deep-learning convention), implicit GEMM: M = pixels, N = Cout,
// K = 9 * Cpad.  CT output channels per CTA (64, or 32 for the 32-channel
// layers); 128 threads: warp w owns pixels 32 (w & 1) + [0, 32) and channels
// (CT / 2) (w >> 1) + [0, CT / 2) of the CTA tile.
template <int CT>
__global__ void __launch_bounds__(128) conv3x3_kernel(ConvArgs a) {
  constexpr int NB = CT / 16;   // n8 blocks per warp
  extern __shared__ __align__(16) unsigned char conv_sm[];
  bf16* halo = reinterpret_cast<bf16*>(conv_sm);                 // [100][kPitch]
  bf16* wsm = halo + kHalo * kHalo * kPitch;                      // [CT][9][kPitch]
  const int tiles_x = (a.W + 7) >> 3;
  const int ty0 = (blockIdx.x / tiles_x) * 8, tx0 = (blockIdx.x % tiles_x) * 8;
  const int n = blockIdx.y, co0 = blockIdx.z * CT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ph = warp & 1, chf = warp >> 1;
  float acc[2][NB][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
  for (int cc = 0; cc < a.Cpad; cc += kCK) {
    for (int t = threadIdx.x; t < kHalo * kHalo * 4; t += blockDim.x) {
      const int hp = t >> 2, g = t & 3;
      const int hy = hp / kHalo, hx = hp - hy * kHalo;
      *reinterpret_cast<uint4*>(halo + hp * kPitch + g * 8) = load_in8(a, n, ty0 + hy - 1, tx0 + hx - 1, cc + g * 8);
    }
    for (int t = threadIdx.x; t < CT * 9 * 4; t += blockDim.x) {
      const int g = t & 3, row = t >> 2;   // row = co_local * 9 + tap
      const int col = row / 9, tap = row - col * 9;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (co0 + col < a.Cout)
        v = *reinterpret_cast<const uint4*>(a.w + ((size_t)(co0 + col) * 9 + tap) * a.Cpad + cc + g * 8);
      *reinterpret_cast<uint4*>(wsm + row * kPitch + g * 8) = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
      const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        unsigned af[2][4];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const int p = ph * 32 + mb * 16 + (lane & 15);
          const int r = p >> 3, c = p & 7;
          ldsm_x4(af[mb], halo + ((r + dy) * kHalo + (c + dx)) * kPitch + ks * 16 + (lane >> 4) * 8);
        }
        unsigned bfr[NB / 2][4];
#pragma unroll
        for (int np = 0; np < NB / 2; ++np) {
          const int mi = lane >> 3;
          const int co = chf * (CT / 2) + np * 16 + ((mi >> 1) << 3) + (lane & 7);
          ldsm_x4(bfr[np], wsm + (co * 9 + tap) * kPitch + ks * 16 + (mi & 1) * 8);
        }
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
          for (int nb = 0; nb < NB; ++nb)
            mma_bf16(acc[mb][nb], af[mb], bfr[nb >> 1][(nb & 1) * 2], bfr[nb >> 1][(nb & 1) * 2 + 1]);
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mb = 0; mb < 2; ++mb)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int p = ph * 32 + mb * 16 + g + half * 8;
      const int y = ty0 + (p >> 3), x = tx0 + (p & 7);
      if (y >= a.H || x >= a.W) continue;
      bf16* op = a.out + (((size_t)n * a.H + y) * a.W + x) * a.out_pitch;
#pragma unroll
      for (int nb = 0; nb < NB; ++nb) {
        const int co = co0 + chf * (CT / 2) + nb * 8 + 2 * tq;
        float v0 = acc[mb][nb][half * 2], v1 = acc[mb][nb][half * 2 + 1];
        if (a.bias) {
          if (co < a.Cout) v0 += a.bias[co];
          if (co + 1 < a.Cout) v1 += a.bias[co + 1];
        }
        if (a.relu) {
          v0 = fmaxf(v0, 0.f);
          v1 = fmaxf(v1, 0.f);
        }
        if (co + 1 < a.Cout)
          *reinterpret_cast<__nv_bfloat162*>(op + co) = __floats2bfloat162_rn(v0, v1);
        else if (co < a.Cout)
          op[co] = __float2bfloat16(v0);
      }
    }
}

constexpr size_t kConvSmem = (size_t)(kHalo * kHalo + kCT * 9) * kPitch * sizeof(bf16);   // CT = 64

// Weight gradient of a 3x3 convolution: dW[co][tap][ci] += sum over pixels
// of g[p][co] in[p + offset(tap)][ci].  CTA: 64 output channels x 32 input
// channels x one tap, over a run of 8x8 pixel tiles; warp w owns output
// channels 16 w + [0, 16).
struct WgradArgs {
  ConvArgs in;         // the layer's input description (in0/in1/up/N/H/W/Cin/Cpad/Cout)
  const bf16* g;       // [N][H][W][Cout] gradient at the layer's pre-activation
  float* dw;           // [Cout][9][Cpad] FP32
  int tiles_per_cta;
};

__global__ void __launch_bounds__(128) wgrad_kernel(WgradArgs wa) {
  const ConvArgs& a = wa.in;
  __shared__ __align__(16) bf16 gs[64][72];               // [pixel][64 co + pad]
  __shared__ __align__(16) bf16 hs[kHalo * kHalo][kPitch];  // input halo, 32 channels
  const int ntx = (a.W + 7) >> 3, nty = (a.H + 7) >> 3;
  const int ntiles = a.N * ntx * nty;
  const int tap = blockIdx.y % 9, ccb = blockIdx.y / 9;   // ccb: 32-channel slice of Cpad
  const int co0 = blockIdx.z * kCT;
  const int dy = tap / 3, dx = tap - dy * 3;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[i][k] = 0.f;
  const int t_beg = blockIdx.x * wa.tiles_per_cta, t_end = min(ntiles, t_beg + wa.tiles_per_cta);
  for (int tile = t_beg; tile < t_end; ++tile) {
    const int n = tile / (ntx * nty), rem = tile - n * ntx * nty;
    const int ty0 = (rem / ntx) * 8, tx0 = (rem % ntx) * 8;
    for (int t = threadIdx.x; t < 64 * 8; t += blockDim.x) {   // 64 pixels x 8 groups of 8 channels
      const int p = t >> 3, gq = t & 7;
      const int y = ty0 + (p >> 3), x = tx0 + (p & 7);
      const int co = co0 + gq * 8;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (y < a.H && x < a.W && co < a.Cout) {
        const bf16* src = wa.g + (((size_t)n * a.H + y) * a.W + x) * a.Cout + co;
        if (co + 8 <= a.Cout && (a.Cout & 7) == 0) {
          v = *reinterpret_cast<const uint4*>(src);
        } else {
          bf16 tmp[8];
          for (int k = 0; k < 8; ++k) tmp[k] = co + k < a.Cout ? src[k] : __float2bfloat16(0.f);
          v = *reinterpret_cast<const uint4*>(tmp);
        }
      }
      *reinterpret_cast<uint4*>(&gs[p][gq * 8]) = v;
    }
    for (int t = threadIdx.x; t < kHalo * kHalo * 4; t += blockDim.x) {
      const int hp = t >> 2, gq = t & 3;
      const int hy = hp / kHalo, hx = hp - hy * kHalo;
      *reinterpret_cast<uint4*>(&hs[hp][gq * 8]) = load_in8(a, n, ty0 + hy - 1, tx0 + hx - 1, ccb * kCK + gq * 8);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {   // 64 pixels = 4 x k16
      unsigned af[4];
      {
        const int mi = lane >> 3;
        const int p = ks * 16 + ((mi >> 1) << 3) + (lane & 7);
        const int co = warp * 16 + (mi & 1) * 8;
        ldsm_x4_t(af, &gs[p][co]);
      }
      unsigned bfr[2][4];
#pragma unroll
      for (int np = 0; np < 2; ++np) {
        const int mi = lane >> 3;
        const int p = ks * 16 + (mi & 1) * 8 + (lane & 7);
        const int r = p >> 3, c = p & 7;
        const int ci = np * 16 + (mi >> 1) * 8;
        ldsm_x4_t(bfr[np], &hs[(r + dy) * kHalo + (c + dx)][ci]);
      }
#pragma unroll
      for (int nb = 0; nb < 4; ++nb) mma_bf16(acc[nb], af, bfr[nb >> 1][(nb & 1) * 2], bfr[nb >> 1][(nb & 1) * 2 + 1]);
    }
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int nb = 0; nb < 4; ++nb)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int co = co0 + warp * 16 + g + half * 8;
      const int ci = ccb * kCK + nb * 8 + 2 * tq;
      if (co >= a.Cout) continue;
      float* d = wa.dw + ((size_t)co * 9 + tap) * a.Cpad;
      if (ci < a.Cin) atomicAdd(d + ci, acc[nb][half * 2]);
      if (ci + 1 < a.Cin) atomicAdd(d + ci + 1, acc[nb][half * 2 + 1]);
    }
}

// ----------------------------------------------------------- small kernels
__global__ void image_to_nhwc_kernel(const float* __restrict__ img, const float* __restrict__ scale, int npix,
                                     int nimg, bf16* __restrict__ out) {
  const int64_t n = (int64_t)npix * nimg;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(img[i] * scale[i / npix]);
}

// out[n][y][x] = (sum_c f[p][c] wh[c] + bh) / scale[n]
__global__ void head_fwd_kernel(const bf16* __restrict__ f, int C, const float* __restrict__ wh, const float* bh,
                                const float* __restrict__ img, const float* __restrict__ scale, int npix, int nimg,
                                float* __restrict__ out) {
  const int64_t n = (int64_t)npix * nimg;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float s = bh[0];
    for (int c = 0; c < C; ++c) s = fmaf(__bfloat162float(f[i * C + c]), wh[c], s);
    out[i] = s / scale[i / npix];
  }
}

// loss = mean((out - target)^2) over the normalised outputs; g = d loss / d head output
__global__ void head_bwd_kernel(const bf16* __restrict__ f, int C, const float* __restrict__ wh,
                                const float* __restrict__ out, const float* __restrict__ target,
                                const float* __restrict__ scale, int npix, int nimg, float inv_count,
                                bf16* __restrict__ gf, float* __restrict__ dwh, float* __restrict__ dbh,
                                double* __restrict__ loss) {
  __shared__ float sdw[64];
  __shared__ float sdb;
  __shared__ double sl;
  if (threadIdx.x < 64) sdw[threadIdx.x] = 0.f;
  if (threadIdx.x == 0) {
    sdb = 0.f;
    sl = 0.0;
  }
  __syncthreads();
  float dwl[32];
  for (int c = 0; c < 32; ++c) dwl[c] = 0.f;
  float dbl = 0.f;
  double ll = 0.0;
  const int64_t n = (int64_t)npix * nimg;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float sc = scale[i / npix];
    const float e = (out[i] - target[i]) * sc;   // error of the normalised output
    ll += (double)e * e;
    const float go = 2.f * e * inv_count;        // d loss / d (normalised head output)
    dbl += go;
    for (int c = 0; c < C; ++c) {
      const float fv = __bfloat162float(f[i * C + c]);
      gf[i * C + c] = __float2bfloat16(go * wh[c]);
      if (c < 32) dwl[c] = fmaf(go, fv, dwl[c]);
    }
  }
  for (int c = 0; c < C && c < 32; ++c) atomicAdd(&sdw[c], dwl[c]);
  atomicAdd(&sdb, dbl);
  atomicAdd(&sl, ll);
  __syncthreads();
  if (threadIdx.x < C && threadIdx.x < 32) atomicAdd(dwh + threadIdx.x, sdw[threadIdx.x]);
  if (threadIdx.x == 0) {
    atomicAdd(dbh, sdb);
    atomicAdd(loss, sl * inv_count);
  }
}

__global__ void avgpool_fwd_kernel(const bf16* __restrict__ in, int N, int H, int W, int C, bf16* __restrict__ out) {
  const int h = H >> 1, w = W >> 1;
  const int64_t n = (int64_t)N * h * w * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t pix = i / C;
    const int x = (int)(pix % w), y = (int)((pix / w) % h), b = (int)(pix / ((int64_t)w * h));
    const size_t base = (((size_t)b * H + 2 * y) * W + 2 * x) * C + c;
    const float s = __bfloat162float(in[base]) + __bfloat162float(in[base + C]) +
                    __bfloat162float(in[base + (size_t)W * C]) + __bfloat162float(in[base + (size_t)W * C + C]);
    out[i] = __float2bfloat16(0.25f * s);
  }
}

// g_in (H x W) += g_out(y/2, x/2) / 4   (adjoint of the average pool, accumulated)
__global__ void avgpool_bwd_kernel(const bf16* __restrict__ gout, int N, int H, int W, int C, bf16* __restrict__ gin) {
  const int h = H >> 1, w = W >> 1;
  const int64_t n = (int64_t)N * H * W * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t pix = i / C;
    const int x = (int)(pix % W), y = (int)((pix / W) % H), b = (int)(pix / ((int64_t)W * H));
    const float v = 0.25f * __bfloat162float(gout[(((size_t)b * h + (y >> 1)) * w + (x >> 1)) * C + c]);
    gin[i] = __float2bfloat16(__bfloat162float(gin[i]) + v);
  }
}

// g_low(y, x) = sum of the 2x2 block of g_high (adjoint of the nearest upsample)
__global__ void upsample_bwd_kernel(const bf16* __restrict__ ghigh, int pitch, int N, int H, int W, int C,
                                    bf16* __restrict__ glow) {
  const int h = H >> 1, w = W >> 1;
  const int64_t n = (int64_t)N * h * w * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t pix = i / C;
    const int x = (int)(pix % w), y = (int)((pix / w) % h), b = (int)(pix / ((int64_t)w * h));
    const size_t base = (((size_t)b * H + 2 * y) * W + 2 * x) * pitch + c;
    const float s = __bfloat162float(ghigh[base]) + __bfloat162float(ghigh[base + pitch]) +
                    __bfloat162float(ghigh[base + (size_t)W * pitch]) +
                    __bfloat162float(ghigh[base + (size_t)W * pitch + pitch]);
    glow[i] = __float2bfloat16(s);
  }
}

// g <- g * (y > 0): gradient at the pre-activation of a ReLU layer (g may be
// a channel slice of a wider buffer: pitch)
__global__ void relu_mask_kernel(const bf16* __restrict__ gsrc, int src_pitch, const bf16* __restrict__ y, int C,
                                 int64_t npix, bf16* __restrict__ g) {
  const int64_t n = npix * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i - p * C);
    const float gv = __bfloat162float(gsrc[p * src_pitch + c]);
    g[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.f ? gv : 0.f);
  }
}

// g_dst[p][c] += g_src[p][c] (src a channel slice of a wider buffer)
__global__ void add_slice_kernel(const bf16* __restrict__ src, int src_pitch, int C, int64_t npix,
                                 bf16* __restrict__ dst) {
  const int64_t n = npix * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i - p * C);
    dst[i] = __float2bfloat16(__bfloat162float(dst[i]) + __bfloat162float(src[p * src_pitch + c]));
  }
}

// db[c] += sum_p g[p][c]
__global__ void bias_grad_kernel(const bf16* __restrict__ g, int C, int64_t npix, float* __restrict__ db) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int64_t p = blockIdx.x; p < npix; p += gridDim.x) s += __bfloat162float(g[p * C + c]);
  atomicAdd(db + c, s);
}

// Adam on the flat FP32 parameters
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// forward weights [Cout][9][Cpad] (BF16) from the FP32 [Cout][Cin][3][3]
// parameters, and the data-gradient weights [Cin][9][CoutPad] with the taps
// flipped (tap' = 8 - tap)
__global__ void pack_weights_kernel(const float* __restrict__ w, int Cout, int Cin, int Cpad, int CoutPad,
                                    bf16* __restrict__ wf, bf16* __restrict__ wb) {
  const int64_t n = (int64_t)Cout * 9 * Cpad;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cpad);
    const int tap = (int)((i / Cpad) % 9);
    const int co = (int)(i / ((int64_t)Cpad * 9));
    const float v = ci < Cin ? w[((size_t)co * Cin + ci) * 9 + tap] : 0.f;
    wf[i] = __float2bfloat16(v);
    if (wb && ci < Cin) wb[((size_t)ci * 9 + (8 - tap)) * CoutPad + co] = __float2bfloat16(v);
  }
}

// dW FP32 [Cout][9][Cpad] -> the flat [Cout][Cin][3][3] parameter gradient
__global__ void unpack_wgrad_kernel(const float* __restrict__ dwp, int Cout, int Cin, int Cpad,
                                    float* __restrict__ dw) {
  const int64_t n = (int64_t)Cout * Cin * 9;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int tap = (int)(i % 9);
    const int ci = (int)((i / 9) % Cin);
    const int co = (int)(i / (9 * (int64_t)Cin));
    dw[i] = dwp[((size_t)co * 9 + tap) * Cpad + ci];
  }
}

int nblk(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }
int pad32(int c) { return (c + 31) / 32 * 32; }

}  // namespace

// ------------------------------------------------------------- the network
struct UNetLayer {
  int cin, cout, cpad, coutpad;
  int64_t w_off, b_off;   // offsets into the flat parameter vector
  DevBuf<bf16> wf, wb;    // packed forward / data-gradient weights
  DevBuf<float> dwp;      // weight gradient [Cout][9][Cpad]
};

struct UNet {
  int device = 0;
  cudaStream_t stream = nullptr;
  int base = 32;
  std::vector<std::unique_ptr<UNetLayer>> conv;   // 17 3x3 layers in forward order
  int64_t head_w = 0, head_b = 0, nparam = 0;
  DevBuf<float> param, grad, adam_m, adam_v;
  int64_t adam_t = 0;
  bool packed = false;
  // activations for the current batch
  int N = 0, H = 0, W = 0;
  std::vector<std::unique_ptr<DevBuf<bf16>>> act;
  DevBuf<bf16> xin;
  DevBuf<float> img, tgt, outp, scale;
  DevBuf<double> loss;
  std::vector<std::unique_ptr<DevBuf<bf16>>> gbuf;
  ~UNet() {
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace fhs

using namespace fhs;

namespace {

// Layer order: 0-1 e1, 2-3 e2, 4-5 e3, 6-7 bottleneck, 8 up3, 9-10 d3,
// 11 up2, 12-13 d2, 14 up1, 15-16 d1; head.
struct LayerSpec {
  int cin, cout;
};

std::vector<LayerSpec> layer_specs(int b) {
  return {{1, b},         {b, b},         {b, 2 * b},     {2 * b, 2 * b}, {2 * b, 4 * b},     {4 * b, 4 * b},
          {4 * b, 8 * b}, {8 * b, 8 * b}, {8 * b, 4 * b}, {8 * b, 4 * b}, {4 * b, 4 * b},     {4 * b, 2 * b},
          {4 * b, 2 * b}, {2 * b, 2 * b}, {2 * b, b},     {2 * b, b},     {b, b}};
}

UNet* checked_net(fhs_unet* h) {
  FHS_CHECK(h != nullptr, FHS_ERR_INVALID_ARG, "null network handle");
  return reinterpret_cast<UNet*>(h);
}

template <class F>
fhs_status guarded_unet(F&& f) {
  try {
    f();
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

void pack(UNet* u) {
  if (u->packed) return;
  cudaStream_t s = u->stream;
  for (auto& L : u->conv) {
    const int64_t n = (int64_t)L->cout * 9 * L->cpad;
    pack_weights_kernel<<<nblk(n), 256, 0, s>>>(u->param.p + L->w_off, L->cout, L->cin, L->cpad, L->coutpad, L->wf.p,
                                                L->wb.p);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
  u->packed = true;
}

void conv(UNet* u, const UNetLayer& L, TView in0, TView in1, int up, int N, int H, int W, const bf16* w, int cin,
          int cpad, int cout, const float* bias, int relu, bf16* out, int out_pitch) {
  ConvArgs a;
  a.in0 = in0;
  a.in1 = in1;
  a.up = up;
  a.N = N;
  a.H = H;
  a.W = W;
  a.Cin = cin;
  a.Cpad = cpad;
  a.Cout = cout;
  a.w = w;
  a.bias = bias;
  a.relu = relu;
  a.out = out;
  a.out_pitch = out_pitch;
  (void)L;
  const int ct = cout <= 32 ? 32 : kCT;   // the 32-channel layers use half-width tiles
  dim3 grid(((W + 7) / 8) * ((H + 7) / 8), N, (cout + ct - 1) / ct);
  FHS_CHECK(grid.y <= 65535 && grid.z <= 65535, FHS_ERR_UNSUPPORTED, "batch too large");
  if (ct == 32)
    conv3x3_kernel<32><<<grid, 128, (size_t)(kHalo * kHalo + 32 * 9) * kPitch * sizeof(bf16), u->stream>>>(a);
  else
    conv3x3_kernel<64><<<grid, 128, kConvSmem, u->stream>>>(a);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void wgrad(UNet* u, UNetLayer& L, TView in0, TView in1, int up, int N, int H, int W, const bf16* g) {
  WgradArgs wa;
  wa.in.in0 = in0;
  wa.in.in1 = in1;
  wa.in.up = up;
  wa.in.N = N;
  wa.in.H = H;
  wa.in.W = W;
  wa.in.Cin = L.cin;
  wa.in.Cpad = L.cpad;
  wa.in.Cout = L.cout;
  wa.g = g;
  wa.dw = L.dwp.p;
  const int ntiles = N * ((H + 7) / 8) * ((W + 7) / 8);
  wa.tiles_per_cta = std::max(1, ntiles / 64);
  dim3 grid((ntiles + wa.tiles_per_cta - 1) / wa.tiles_per_cta, 9 * (L.cpad / kCK), (L.cout + kCT - 1) / kCT);
  wgrad_kernel<<<grid, 128, 0, u->stream>>>(wa);
  count_launch();
  FHS_LAUNCH_CHECK();
  // the bias gradient of the same layer
  const int64_t npix = (int64_t)N * H * W;
  bias_grad_kernel<<<dim3(std::min<int64_t>(npix, 1024), (L.cout + 127) / 128), 128, 0, u->stream>>>(
      g, L.cout, npix, u->grad.p + L.b_off);
  count_launch();
  FHS_LAUNCH_CHECK();
}

DevBuf<bf16>& act(UNet* u, int i) { return *u->act[i]; }

// Activation buffers (index: tensor): 0 x (1 ch), 1 e1a, 2 e1, 3 p1, 4 e2a, 5 e2, 6 p2, 7 e3a, 8 e3,
// 9 p3, 10 ba, 11 bb, 12 u3, 13 d3a, 14 d3, 15 u2, 16 d2a, 17 d2, 18 u1, 19 d1a, 20 d1
void ensure_batch(UNet* u, int N, int H, int W) {
  FHS_CHECK(N >= 1 && H >= 8 && W >= 8 && H % 8 == 0 && W % 8 == 0, FHS_ERR_INVALID_ARG,
            "network input: N >= 1 images of H x W, H and W multiples of 8 (>= 8)");
  if (u->N == N && u->H == H && u->W == W) return;
  const int b = u->base;
  const int64_t p0 = (int64_t)N * H * W, p1 = p0 / 4, p2 = p0 / 16, p3 = p0 / 64;
  const int64_t sz[21] = {p0,         p0 * b,     p0 * b,     p1 * b,     p1 * 2 * b, p1 * 2 * b, p2 * 2 * b,
                          p2 * 4 * b, p2 * 4 * b, p3 * 4 * b, p3 * 8 * b, p3 * 8 * b, p2 * 4 * b, p2 * 4 * b,
                          p2 * 4 * b, p1 * 2 * b, p1 * 2 * b, p1 * 2 * b, p0 * b,     p0 * b,     p0 * b};
  u->act.clear();
  for (int i = 0; i < 21; ++i) {
    u->act.emplace_back(new DevBuf<bf16>());
    u->act.back()->alloc(sz[i]);
  }
  u->gbuf.clear();   // gradient scratch, allocated by the first backward pass of this batch size
  u->img.alloc(p0);
  u->tgt.alloc(p0);
  u->outp.alloc(p0);
  u->scale.alloc(N);
  u->N = N;
  u->H = H;
  u->W = W;
}

TView tv(const bf16* p, int C, int pitch = -1) { return TView{p, C, pitch < 0 ? C : pitch}; }

// images (device, [N][H][W] f32, already in u->img) and scales -> u->outp
void forward(UNet* u) {
  pack(u);
  const int N = u->N, H = u->H, W = u->W, b = u->base;
  cudaStream_t s = u->stream;
  const int64_t p0 = (int64_t)N * H * W;
  image_to_nhwc_kernel<<<nblk(p0), 256, 0, s>>>(u->img.p, u->scale.p, H * W, N, act(u, 0).p);
  count_launch();
  auto& C = u->conv;
  auto c3 = [&](int li, TView i0, TView i1, int up, int h, int w, int outi) {
    UNetLayer& L = *C[li];
    conv(u, L, i0, i1, up, N, h, w, L.wf.p, L.cin, L.cpad, L.cout, u->param.p + L.b_off, 1, act(u, outi).p, L.cout);
  };
  auto pool = [&](int ini, int h, int w, int c, int outi) {
    avgpool_fwd_kernel<<<nblk((int64_t)N * h * w * c / 4), 256, 0, s>>>(act(u, ini).p, N, h, w, c, act(u, outi).p);
    count_launch();
    FHS_LAUNCH_CHECK();
  };
  const TView none{nullptr, 0, 0};
  c3(0, tv(act(u, 0).p, 1), none, 0, H, W, 1);
  c3(1, tv(act(u, 1).p, b), none, 0, H, W, 2);
  pool(2, H, W, b, 3);
  c3(2, tv(act(u, 3).p, b), none, 0, H / 2, W / 2, 4);
  c3(3, tv(act(u, 4).p, 2 * b), none, 0, H / 2, W / 2, 5);
  pool(5, H / 2, W / 2, 2 * b, 6);
  c3(4, tv(act(u, 6).p, 2 * b), none, 0, H / 4, W / 4, 7);
  c3(5, tv(act(u, 7).p, 4 * b), none, 0, H / 4, W / 4, 8);
  pool(8, H / 4, W / 4, 4 * b, 9);
  c3(6, tv(act(u, 9).p, 4 * b), none, 0, H / 8, W / 8, 10);
  c3(7, tv(act(u, 10).p, 8 * b), none, 0, H / 8, W / 8, 11);
  c3(8, tv(act(u, 11).p, 8 * b), none, 1, H / 4, W / 4, 12);                       // up3
  c3(9, tv(act(u, 12).p, 4 * b), tv(act(u, 8).p, 4 * b), 0, H / 4, W / 4, 13);    // cat(u3, e3)
  c3(10, tv(act(u, 13).p, 4 * b), none, 0, H / 4, W / 4, 14);
  c3(11, tv(act(u, 14).p, 4 * b), none, 1, H / 2, W / 2, 15);                      // up2
  c3(12, tv(act(u, 15).p, 2 * b), tv(act(u, 5).p, 2 * b), 0, H / 2, W / 2, 16);
  c3(13, tv(act(u, 16).p, 2 * b), none, 0, H / 2, W / 2, 17);
  c3(14, tv(act(u, 17).p, 2 * b), none, 1, H, W, 18);                             // up1
  c3(15, tv(act(u, 18).p, b), tv(act(u, 2).p, b), 0, H, W, 19);
  c3(16, tv(act(u, 19).p, b), none, 0, H, W, 20);
  head_fwd_kernel<<<nblk(p0), 256, 0, s>>>(act(u, 20).p, b, u->param.p + u->head_w, u->param.p + u->head_b,
                                           u->img.p, u->scale.p, H * W, N, u->outp.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

// loss and parameter gradients (u->grad) for targets in u->tgt, after forward()
void backward(UNet* u) {
  const int N = u->N, H = u->H, W = u->W, b = u->base;
  cudaStream_t s = u->stream;
  const int64_t p0 = (int64_t)N * H * W;
  if (u->gbuf.empty()) {   // four maps of 2b channels at full size cover every gradient and concat
    for (int i = 0; i < 4; ++i) {
      u->gbuf.emplace_back(new DevBuf<bf16>());
      u->gbuf.back()->alloc(p0 * 2 * b);
    }
  }
  u->grad.zero(s);
  for (auto& L : u->conv) L->dwp.zero(s);
  u->loss.zero(s);
  bf16* g0 = u->gbuf[0]->p;   // gradient at a layer output / pre-activation (ping)
  bf16* g1 = u->gbuf[1]->p;   // pong
  bf16* gc = u->gbuf[2]->p;   // data gradient of a conv input (possibly a concat)
  bf16* gs = u->gbuf[3]->p;   // skip-connection gradients awaiting their encoder layer
  head_bwd_kernel<<<std::min<int64_t>((p0 + 255) / 256, 1024), 256, 0, s>>>(
      act(u, 20).p, b, u->param.p + u->head_w, u->outp.p, u->tgt.p, u->scale.p, H * W, N, 1.f / (float)p0, g0,
      u->grad.p + u->head_w, u->grad.p + u->head_b, u->loss.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  auto& C = u->conv;
  const TView none{nullptr, 0, 0};
  auto mask = [&](const bf16* gsrc, int pitch, int yi, int c, int64_t np, bf16* dst) {
    relu_mask_kernel<<<nblk(np * c), 256, 0, s>>>(gsrc, pitch, act(u, yi).p, c, np, dst);
    count_launch();
    FHS_LAUNCH_CHECK();
  };
  // one conv layer backward: gpre = mask(gout); wgrad; data gradient into gin (if needed)
  auto layer = [&](int li, const bf16* gout, int gpitch, int yi, TView i0, TView i1, int up, int h, int w,
                   bf16* gpre, bf16* gin) {
    UNetLayer& L = *C[li];
    const int64_t np = (int64_t)N * h * w;
    mask(gout, gpitch, yi, L.cout, np, gpre);
    wgrad(u, L, i0, i1, up, N, h, w, gpre);
    if (gin) conv(u, L, tv(gpre, L.cout), none, 0, N, h, w, L.wb.p, L.cout, L.coutpad, L.cin, nullptr, 0, gin, L.cin);
  };
  auto upb = [&](const bf16* gh, int pitch, int h, int w, int c, bf16* gl) {   // (h, w): high-res size
    upsample_bwd_kernel<<<nblk((int64_t)N * h * w * c / 4), 256, 0, s>>>(gh, pitch, N, h, w, c, gl);
    count_launch();
    FHS_LAUNCH_CHECK();
  };
  auto poolb = [&](const bf16* gl, int h, int w, int c, bf16* gh) {   // accumulate into gh (h, w high-res)
    avgpool_bwd_kernel<<<nblk((int64_t)N * h * w * c), 256, 0, s>>>(gl, N, h, w, c, gh);
    count_launch();
    FHS_LAUNCH_CHECK();
  };
  auto addsl = [&](const bf16* src, int pitch, int c, int64_t np, bf16* dst) {
    add_slice_kernel<<<nblk(np * c), 256, 0, s>>>(src, pitch, c, np, dst);
    count_launch();
    FHS_LAUNCH_CHECK();
  };
  auto copy = [&](const bf16* src, int pitch, int c, int64_t np, bf16* dst) {
    FHS_CUDA(cudaMemsetAsync(dst, 0, np * c * sizeof(bf16), s));
    addsl(src, pitch, c, np, dst);
  };
  const int64_t q0 = p0, q1 = p0 / 4, q2 = p0 / 16, q3 = p0 / 64;
  // d1: 16 (in d1a), 15 (in cat(u1, e1))
  layer(16, g0, b, 20, tv(act(u, 19).p, b), none, 0, H, W, g1, gc);
  layer(15, gc, b, 19, tv(act(u, 18).p, b), tv(act(u, 2).p, b), 0, H, W, g1, gc);   // gc: [u1 | e1]
  copy(gc + b, 2 * b, b, q0, gs);                                    // skip gradient of e1 (kept in gs, level 1)
  layer(14, gc, 2 * b, 18, tv(act(u, 17).p, 2 * b), none, 1, H, W, g1, g0);        // up1: data grad at full res
  upb(g0, 2 * b, H, W, 2 * b, g1);                                                   // -> d2 (H/2)
  // d2
  layer(13, g1, 2 * b, 17, tv(act(u, 16).p, 2 * b), none, 0, H / 2, W / 2, g0, gc);
  layer(12, gc, 2 * b, 16, tv(act(u, 15).p, 2 * b), tv(act(u, 5).p, 2 * b), 0, H / 2, W / 2, g0, gc);
  bf16* gs2 = gs + q0 * b;   // level-2 skip gradient after the level-1 one
  copy(gc + 2 * b, 4 * b, 2 * b, q1, gs2);
  layer(11, gc, 4 * b, 15, tv(act(u, 14).p, 4 * b), none, 1, H / 2, W / 2, g0, g1);
  upb(g1, 4 * b, H / 2, W / 2, 4 * b, g0);                                           // -> d3 (H/4)
  // d3
  layer(10, g0, 4 * b, 14, tv(act(u, 13).p, 4 * b), none, 0, H / 4, W / 4, g1, gc);
  layer(9, gc, 4 * b, 13, tv(act(u, 12).p, 4 * b), tv(act(u, 8).p, 4 * b), 0, H / 4, W / 4, g1, gc);
  bf16* gs3 = gs2 + q1 * 2 * b;
  copy(gc + 4 * b, 8 * b, 4 * b, q2, gs3);
  layer(8, gc, 8 * b, 12, tv(act(u, 11).p, 8 * b), none, 1, H / 4, W / 4, g1, g0);
  upb(g0, 8 * b, H / 4, W / 4, 8 * b, g1);                                           // -> bb (H/8)
  // bottleneck
  layer(7, g1, 8 * b, 11, tv(act(u, 10).p, 8 * b), none, 0, H / 8, W / 8, g0, gc);
  layer(6, gc, 8 * b, 10, tv(act(u, 9).p, 4 * b), none, 0, H / 8, W / 8, g0, gc);   // gc: grad of p3
  // e3 = skip + pool adjoint
  poolb(gc, H / 4, W / 4, 4 * b, gs3);
  layer(5, gs3, 4 * b, 8, tv(act(u, 7).p, 4 * b), none, 0, H / 4, W / 4, g0, gc);
  layer(4, gc, 4 * b, 7, tv(act(u, 6).p, 2 * b), none, 0, H / 4, W / 4, g0, gc);    // grad of p2
  poolb(gc, H / 2, W / 2, 2 * b, gs2);
  layer(3, gs2, 2 * b, 5, tv(act(u, 4).p, 2 * b), none, 0, H / 2, W / 2, g0, gc);
  layer(2, gc, 2 * b, 4, tv(act(u, 3).p, b), none, 0, H / 2, W / 2, g0, gc);        // grad of p1
  poolb(gc, H, W, b, gs);
  layer(1, gs, b, 2, tv(act(u, 1).p, b), none, 0, H, W, g0, gc);
  layer(0, gc, b, 1, tv(act(u, 0).p, 1), none, 0, H, W, g0, nullptr);
  (void)q3;
  for (auto& L : u->conv) {
    const int64_t n = (int64_t)L->cout * L->cin * 9;
    unpack_wgrad_kernel<<<nblk(n), 256, 0, s>>>(L->dwp.p, L->cout, L->cin, L->cpad, u->grad.p + L->w_off);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
}

// host images -> device, per-image normalisation 1 / max |x| (1 if zero)
void load_images(UNet* u, int N, int H, int W, const float* img, const float* tgt) {
  ensure_batch(u, N, H, W);
  cudaStream_t s = u->stream;
  const int64_t np = (int64_t)H * W;
  std::vector<float> sc(N, 1.f);
  for (int n = 0; n < N; ++n) {
    float m = 0.f;
    for (int64_t i = 0; i < np; ++i) m = std::max(m, std::fabs(img[n * np + i]));
    FHS_CHECK(std::isfinite(m), FHS_ERR_NUMERIC, "non-finite network input");
    sc[n] = m > 0.f ? 1.f / m : 1.f;
  }
  u->img.upload(img, N * np, s);
  if (tgt) u->tgt.upload(tgt, N * np, s);
  u->scale.upload(sc.data(), N, s);
}

}  // namespace

namespace fhs {

// input scale 1 / max|image| per image (1 for an all-zero image), one CTA
// per image, as load_images does on the host
__global__ void unet_image_scale_kernel(const float* __restrict__ img, int64_t np, float* __restrict__ scale) {
  __shared__ float red[256];
  const float* p = img + (size_t)blockIdx.x * np;
  float m = 0.f;
  for (int64_t i = threadIdx.x; i < np; i += blockDim.x) m = fmaxf(m, fabsf(p[i]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) scale[blockIdx.x] = red[0] > 0.f ? 1.f / red[0] : 1.f;
}

void unet_forward_device(fhs_unet* h, int n, int H, int W, const float* d_img, float* d_out) {
  UNet* u = checked_net(h);
  FHS_CHECK(n >= 1 && d_img && d_out, FHS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard g(u->device);
  ensure_batch(u, n, H, W);
  const int64_t np = (int64_t)H * W;
  FHS_CUDA(cudaMemcpyAsync(u->img.p, d_img, (size_t)n * np * sizeof(float), cudaMemcpyDeviceToDevice, u->stream));
  unet_image_scale_kernel<<<n, 256, 0, u->stream>>>(u->img.p, np, u->scale.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  forward(u);
  FHS_CUDA(cudaMemcpyAsync(d_out, u->outp.p, (size_t)n * np * sizeof(float), cudaMemcpyDeviceToDevice, u->stream));
  FHS_CUDA(cudaStreamSynchronize(u->stream));
}

int unet_device(const fhs_unet* h) { return checked_net(const_cast<fhs_unet*>(h))->device; }

}  // namespace fhs

extern "C" {

fhs_status fhs_unet_create(int device, int base_channels, fhs_unet** out) {
  return guarded_unet([&] {
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    FHS_CHECK(base_channels == 32, FHS_ERR_UNSUPPORTED, "this build's network has 32 base channels");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(FHS_ERR_NO_DEVICE, "no CUDA device");
    FHS_CHECK(device >= 0 && device < ndev, FHS_ERR_INVALID_ARG, "bad device index");
    DeviceGuard g(device);
    std::unique_ptr<UNet> u(new UNet());
    u->device = device;
    u->base = base_channels;
    FHS_CUDA(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking));
    FHS_CUDA(cudaFuncSetAttribute(conv3x3_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvSmem));
    int64_t off = 0;
    for (const auto& sp : layer_specs(base_channels)) {
      std::unique_ptr<UNetLayer> L(new UNetLayer());
      L->cin = sp.cin;
      L->cout = sp.cout;
      L->cpad = pad32(sp.cin);
      L->coutpad = pad32(sp.cout);
      L->w_off = off;
      off += (int64_t)sp.cout * sp.cin * 9;
      L->b_off = off;
      off += sp.cout;
      L->wf.alloc((size_t)L->cout * 9 * L->cpad);
      L->wb.alloc((size_t)L->cin * 9 * L->coutpad);
      L->wb.zero(u->stream);
      L->dwp.alloc((size_t)L->cout * 9 * L->cpad);
      u->conv.push_back(std::move(L));
    }
    u->head_w = off;
    off += base_channels;
    u->head_b = off;
    off += 1;
    u->nparam = off;
    u->param.alloc(off);
    u->param.zero(u->stream);
    u->grad.alloc(off);
    u->adam_m.alloc(off);
    u->adam_v.alloc(off);
    u->adam_m.zero(u->stream);
    u->adam_v.zero(u->stream);
    u->loss.alloc(1);
    FHS_CUDA(cudaStreamSynchronize(u->stream));
    *out = reinterpret_cast<fhs_unet*>(u.release());
  });
}

fhs_status fhs_unet_destroy(fhs_unet* h) {
  return guarded_unet([&] {
    if (!h) return;
    UNet* u = reinterpret_cast<UNet*>(h);
    DeviceGuard g(u->device);
    cudaStreamSynchronize(u->stream);
    delete u;
  });
}

int64_t fhs_unet_n_params(const fhs_unet* h) {
  return h ? reinterpret_cast<const UNet*>(h)->nparam : -1;
}

fhs_status fhs_unet_set_params(fhs_unet* h, const float* params) {
  return guarded_unet([&] {
    UNet* u = checked_net(h);
    FHS_CHECK(params != nullptr, FHS_ERR_INVALID_ARG, "null parameters");
    for (int64_t i = 0; i < u->nparam; ++i) FHS_CHECK(std::isfinite(params[i]), FHS_ERR_NUMERIC, "non-finite parameter");
    DeviceGuard g(u->device);
    u->param.upload(params, u->nparam, u->stream);
    u->adam_m.zero(u->stream);
    u->adam_v.zero(u->stream);
    u->adam_t = 0;
    u->packed = false;
    FHS_CUDA(cudaStreamSynchronize(u->stream));
  });
}

fhs_status fhs_unet_get_params(fhs_unet* h, float* params) {
  return guarded_unet([&] {
    UNet* u = checked_net(h);
    FHS_CHECK(params != nullptr, FHS_ERR_INVALID_ARG, "null output");
    DeviceGuard g(u->device);
    u->param.download(params, u->nparam, u->stream);
    FHS_CUDA(cudaStreamSynchronize(u->stream));
  });
}

fhs_status fhs_unet_forward(fhs_unet* h, int n_images, int H, int W, const float* images, float* out) {
  return guarded_unet([&] {
    UNet* u = checked_net(h);
    FHS_CHECK(images && out, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(u->device);
    load_images(u, n_images, H, W, images, nullptr);
    forward(u);
    u->outp.download(out, (size_t)n_images * H * W, u->stream);
    FHS_CUDA(cudaStreamSynchronize(u->stream));
  });
}

fhs_status fhs_unet_gradient(fhs_unet* h, int n_images, int H, int W, const float* images, const float* targets,
                             float* grad, double* loss) {
  return guarded_unet([&] {
    UNet* u = checked_net(h);
    FHS_CHECK(images && targets, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(u->device);
    load_images(u, n_images, H, W, images, targets);
    forward(u);
    backward(u);
    if (grad) u->grad.download(grad, u->nparam, u->stream);
    if (loss) u->loss.download(loss, 1, u->stream);
    FHS_CUDA(cudaStreamSynchronize(u->stream));
  });
}

fhs_status fhs_unet_train_step(fhs_unet* h, int n_images, int H, int W, const float* images, const float* targets,
                               float lr, double* loss) {
  return guarded_unet([&] {
    UNet* u = checked_net(h);
    FHS_CHECK(images && targets, FHS_ERR_INVALID_ARG, "null buffer");
    FHS_CHECK(std::isfinite(lr) && lr > 0.f, FHS_ERR_INVALID_ARG, "learning rate must be finite and > 0");
    DeviceGuard g(u->device);
    load_images(u, n_images, H, W, images, targets);
    forward(u);
    backward(u);
    ++u->adam_t;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)u->adam_t));
    const float c2 = 1.f / (1.f - std::pow(b2, (float)u->adam_t));
    adam_kernel<<<nblk(u->nparam), 256, 0, u->stream>>>(u->param.p, u->grad.p, u->adam_m.p, u->adam_v.p, u->nparam,
                                                         lr, b1, b2, eps, c1, c2);
    count_launch();
    FHS_LAUNCH_CHECK();
    u->packed = false;
    if (loss) u->loss.download(loss, 1, u->stream);
    FHS_CUDA(cudaStreamSynchronize(u->stream));
  });
}

}  // extern "C"
