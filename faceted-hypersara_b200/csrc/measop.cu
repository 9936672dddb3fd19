// Measurement operator Phi_l = G_l A on B200 (sm_100a).
//
// Replaces op_p_nufft / A / At / G of the RI-measurement-operator submodule as
// applied by src/update_dual_data_fidelity.m:116-147,
// lib/operators/HS_forward_operator_G.m:36-52 and HS_adjoint_operator_G.m:42-57.
//
// Layout in HBM (per channel l, planes contiguous):
//   image  x[l][ix][iy]          f32  (MATLAB column-major, y fastest)
//   grids  pad/A/B[l][kx][ky]    c64  (Ky = oy*Ny fastest)
//   visibilities, sorted by (tile, sub-bin): geom (f32 fy, f32 fx, u32 kpack,
//   f32 weight), y / v2 / GFx_old c64.
// The image is placed at (n - N/2) mod K before the FFT, which moves the
// reference's centring phase exp(i om N/2) out of G: every tap coefficient is
// then a function of the fractional grid offset only, evaluated from degree-8
// polynomials fitted (FP64, host) to the exact min-max coefficients.
//
// The l2-ball dual takes two passes because the block norm ||z_b|| is a
// reduction over all of a block's visibilities: pass 1 writes z to a scratch
// buffer (zbuf) that pass 2 reads while the owner tile writes v2 = z*scale, so
// CTAs that read a neighbour's visibilities never see a half-updated v2.
//
// Degridding: one CTA per 64x64 grid tile stages the tile and its (J-1)-cell
// apron in shared memory and gathers the taps of the visibilities that start
// in the tile.  Gridding: one CTA per tile accumulates, in shared memory, the
// taps of the visibilities that start in the tile or in the 8-cell ring below
// it, then writes the tile once: no global atomics, no grid zeroing.
#include "measop.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace fhs {

unsigned long long g_launches = 0;

namespace {

constexpr int kS = kTableSamples;
constexpr int kSmemPitch = kTileCells + kBinCells;  // 72 (>= 64 + J - 1)

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // conj(a) * b
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {  // a*b + c
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// Tap coefficients h_j(f) of one axis by Horner evaluation of degree-8
// polynomials in f - 1/2 (FP32, < 1e-7 relative to the FP64 construction).
template <int J>
__device__ __forceinline__ void taps(const float (&P)[kMaxTaps][2][kPolyDegree + 1], float f, float2 (&h)[J]) {
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

__device__ __forceinline__ int wrap(int k, int K) {
  k %= K;
  return k < 0 ? k + K : k;
}

// ---------------------------------------------------------------- degrid
template <int J, bool DUAL>
__global__ void __launch_bounds__(256) degrid_kernel(OpView op, const float2* __restrict__ grid, int c0,
                                                     float2* __restrict__ out, const float2* __restrict__ v2,
                                                     float2* __restrict__ gold,
                                                     const float2* __restrict__ y,
                                                     double* __restrict__ partials, float2* __restrict__ zbuf) {
  // pitch 72 along y: starts within a sub-bin spread over distinct bank pairs
  constexpr int P = kSmemPitch;
  constexpr int R = kTileCells + J - 1;
  __shared__ float2 sm[R * P];
  __shared__ double bacc[kMaxBlocksPerChannel * 2];
  const int tile = blockIdx.x;
  const int ch = c0 + blockIdx.y;
  const int t0 = tile % op.nT0, t1 = tile / op.nT0;
  const int32_t* off = op.sb_off + (size_t)ch * (op.nkeys + 1);
  const int beg = off[tile * kSubPerTile * kSubPerTile];
  const int end = off[(tile + 1) * kSubPerTile * kSubPerTile];
  if (DUAL) {
    if (threadIdx.x < kMaxBlocksPerChannel * 2) bacc[threadIdx.x] = 0.0;
  }
  if (beg == end) {
    if (DUAL && threadIdx.x < kMaxBlocksPerChannel * 2)
      partials[((size_t)blockIdx.y * gridDim.x + tile) * kMaxBlocksPerChannel * 2 + threadIdx.x] = 0.0;
    return;
  }
  const int a0 = t0 * kTileCells, a1 = t1 * kTileCells;
  const float2* g = grid + (size_t)ch * op.Ky * op.Kx;
  for (int idx = threadIdx.x; idx < R * R; idx += blockDim.x) {
    const int c1 = idx / R, cc0 = idx - c1 * R;
    const int k0 = wrap(a0 + cc0, op.Ky), k1 = wrap(a1 + c1, op.Kx);
    sm[c1 * P + cc0] = __ldg(g + (size_t)k1 * op.Ky + k0);
  }
  __syncthreads();
  const int64_t vo = op.ch_voff[ch];
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const float4 gm = __ldg(op.geom + vo + i);
    const unsigned kp = __float_as_uint(gm.z);
    const int d0 = (int)(kp & 0x3FFFu) - a0;
    const int d1 = (int)((kp >> 14) & 0x3FFFu) - a1;
    float2 hy[J], hx[J];
    taps<J>(op.py, gm.x, hy);
    taps<J>(op.px, gm.y, hx);
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int jx = 0; jx < J; ++jx) {
      const float2* col = sm + (d1 + jx) * P + d0;
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int jy = 0; jy < J; ++jy) s = cfma(hy[jy], col[jy], s);
      acc = cfma(hx[jx], s, acc);
    }
    const float2 gfx = make_float2(gm.w * acc.x, gm.w * acc.y);
    if (!DUAL) {
      out[vo + i] = gfx;
    } else {
      const float2 yv = y[vo + i];
      const float2 vv = v2[vo + i];
      const float2 go = gold[vo + i];
      const float2 z = make_float2(vv.x + 2.f * gfx.x - go.x - yv.x, vv.y + 2.f * gfx.y - go.y - yv.y);
      const float2 r = make_float2(gfx.x - yv.x, gfx.y - yv.y);
      zbuf[vo + i] = z;
      gold[vo + i] = gfx;
      const int blk = (int)(kp >> 28);
      atomicAdd(&bacc[2 * blk], (double)z.x * z.x + (double)z.y * z.y);
      atomicAdd(&bacc[2 * blk + 1], (double)r.x * r.x + (double)r.y * r.y);
    }
  }
  if (DUAL) {
    __syncthreads();
    if (threadIdx.x < kMaxBlocksPerChannel * 2)
      partials[((size_t)blockIdx.y * gridDim.x + tile) * kMaxBlocksPerChannel * 2 + threadIdx.x] =
          bacc[threadIdx.x];
  }
}

// ------------------------------------------------------------------ grid
struct Range {
  int beg, end;
  int ring0, ring1;
};

__device__ __forceinline__ int sb_key(const OpView& op, int sb0, int sb1) {
  return ((sb1 / kSubPerTile) * op.nT0 + sb0 / kSubPerTile) * (kSubPerTile * kSubPerTile) +
         (sb1 % kSubPerTile) * kSubPerTile + (sb0 % kSubPerTile);
}

template <int J, bool DUAL>
__global__ void __launch_bounds__(256) grid_kernel(OpView op, float2* __restrict__ gridB, int c0,
                                                   const float2* __restrict__ vin,
                                                   float2* __restrict__ v2,
                                                   const float* __restrict__ blk_scale,
                                                   const float2* __restrict__ zbuf) {
  __shared__ float acc_re[kTileCells * kSmemPitch];
  __shared__ float acc_im[kTileCells * kSmemPitch];
  __shared__ Range rng[2 + 2 * kSubPerTile];
  __shared__ int nrng;
  __shared__ int total;
  const int tile = blockIdx.x;
  const int ch = c0 + blockIdx.y;
  const int t0 = tile % op.nT0, t1 = tile / op.nT0;
  const int a0 = t0 * kTileCells, a1 = t1 * kTileCells;
  const int T0 = min(kTileCells, op.Ky - a0), T1 = min(kTileCells, op.Kx - a1);
  const int32_t* off = op.sb_off + (size_t)ch * (op.nkeys + 1);
  for (int i = threadIdx.x; i < kTileCells * kSmemPitch; i += blockDim.x) {
    acc_re[i] = 0.f;
    acc_im[i] = 0.f;
  }
  if (threadIdx.x == 0) {
    int n = 0;
    const int kb = tile * kSubPerTile * kSubPerTile;
    rng[n++] = Range{off[kb], off[kb + kSubPerTile * kSubPerTile], 0, 0};
    const int sbc0 = (t0 * kSubPerTile - 1 + op.nsb0) % op.nsb0;
    const int sbr1 = (t1 * kSubPerTile - 1 + op.nsb1) % op.nsb1;
    const int sb1_end = min(t1 * kSubPerTile + kSubPerTile, op.nsb1);
    const int sb0_end = min(t0 * kSubPerTile + kSubPerTile, op.nsb0);
    for (int sb1 = t1 * kSubPerTile; sb1 < sb1_end; ++sb1) {
      const int k = sb_key(op, sbc0, sb1);
      if (off[k + 1] > off[k]) rng[n++] = Range{off[k], off[k + 1], 1, 0};
    }
    {
      const int k = sb_key(op, t0 * kSubPerTile, sbr1);
      const int k2 = sb_key(op, sb0_end - 1, sbr1) + 1;
      if (off[k2] > off[k]) rng[n++] = Range{off[k], off[k2], 0, 1};
    }
    {
      const int k = sb_key(op, sbc0, sbr1);
      if (off[k + 1] > off[k]) rng[n++] = Range{off[k], off[k + 1], 1, 1};
    }
    int tot = 0;
    for (int r = 0; r < n; ++r) tot += rng[r].end - rng[r].beg;
    nrng = n;
    total = tot;
  }
  __syncthreads();
  const int64_t vo = op.ch_voff[ch];
  const float* scl = DUAL ? blk_scale + (size_t)ch * kMaxBlocksPerChannel : nullptr;
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    int r = 0, rem = it;
    while (rem >= rng[r].end - rng[r].beg) {
      rem -= rng[r].end - rng[r].beg;
      ++r;
    }
    const int i = rng[r].beg + rem;
    const float4 gm = __ldg(op.geom + vo + i);
    const unsigned kp = __float_as_uint(gm.z);
    int d0 = (int)(kp & 0x3FFFu) - a0;
    int d1 = (int)((kp >> 14) & 0x3FFFu) - a1;
    if (rng[r].ring0 && d0 >= 0) d0 -= op.Ky;
    if (rng[r].ring1 && d1 >= 0) d1 -= op.Kx;
    const bool own = (r == 0);
    float2 v;
    if (DUAL) {
      const float2 z = zbuf[vo + i];
      const float sc = scl[kp >> 28];
      v = make_float2(z.x * sc, z.y * sc);
      if (own) v2[vo + i] = v;
    } else {
      v = vin[vo + i];
    }
    if (d0 + J <= 0 || d0 >= T0 || d1 + J <= 0 || d1 >= T1) continue;
    float2 hy[J], hx[J];
    taps<J>(op.py, gm.x, hy);
    taps<J>(op.px, gm.y, hx);
    v.x *= gm.w;
    v.y *= gm.w;
#pragma unroll
    for (int jx = 0; jx < J; ++jx) {
      const int c1 = d1 + jx;
      if ((unsigned)c1 >= (unsigned)T1) continue;
      const float2 t = cmulc(hx[jx], v);
#pragma unroll
      for (int jy = 0; jy < J; ++jy) {
        const int cc0 = d0 + jy;
        if ((unsigned)cc0 >= (unsigned)T0) continue;
        const float2 a = cmulc(hy[jy], t);
        atomicAdd(&acc_re[c1 * kSmemPitch + cc0], a.x);
        atomicAdd(&acc_im[c1 * kSmemPitch + cc0], a.y);
      }
    }
  }
  __syncthreads();
  float2* gb = gridB + (size_t)ch * op.Ky * op.Kx;
  for (int idx = threadIdx.x; idx < T0 * T1; idx += blockDim.x) {
    const int c1 = idx / T0, cc0 = idx - c1 * T0;
    gb[(size_t)(a1 + c1) * op.Ky + a0 + cc0] =
        make_float2(acc_re[c1 * kSmemPitch + cc0], acc_im[c1 * kSmemPitch + cc0]);
  }
}

// ------------------------------------------------------- pad / crop / misc
__global__ void pad_kernel(const float* __restrict__ x, float2* __restrict__ pad, const float* __restrict__ sy,
                           const float* __restrict__ sx, int Ny, int Nx, int Ky, int Kx, int p0) {
  const int64_t N = (int64_t)Ny * Nx;
  const int plane = blockIdx.y;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(p / Ny), iy = (int)(p - (int64_t)ix * Ny);
    int ky = iy - Ny / 2;
    ky += ky < 0 ? Ky : 0;
    int kx = ix - Nx / 2;
    kx += kx < 0 ? Kx : 0;
    const float v = x[(size_t)plane * N + p] * sy[iy] * sx[ix];
    pad[(size_t)(p0 + plane) * Ky * Kx + (size_t)kx * Ky + ky] = make_float2(v, 0.f);
  }
}

__global__ void crop_real_kernel(const float2* __restrict__ grid, float* __restrict__ out,
                                 const float* __restrict__ sigma, const float* __restrict__ sy,
                                 const float* __restrict__ sx, int Ny, int Nx, int Ky, int Kx, int p0) {
  const int64_t N = (int64_t)Ny * Nx;
  const int plane = blockIdx.y;
  const float sg = sigma ? sigma[plane] : 1.f;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(p / Ny), iy = (int)(p - (int64_t)ix * Ny);
    int ky = iy - Ny / 2;
    ky += ky < 0 ? Ky : 0;
    int kx = ix - Nx / 2;
    kx += kx < 0 ? Kx : 0;
    const float2 g = grid[(size_t)(p0 + plane) * Ky * Kx + (size_t)kx * Ky + ky];
    out[(size_t)plane * N + p] = sg * sy[iy] * sx[ix] * g.x;
  }
}

__global__ void block_reduce_kernel(const double* __restrict__ partials, int ntiles, int c0,
                                    const int32_t* __restrict__ ch_nblk, const int32_t* __restrict__ ch_blkoff,
                                    const double* __restrict__ blk_eps, float* __restrict__ blk_scale,
                                    double* __restrict__ blk_stats) {
  const int c = blockIdx.x;  // relative channel
  const int ch = c0 + c;
  const int b = blockIdx.y;
  if (b >= ch_nblk[ch]) return;
  __shared__ double s0[256], s1[256];
  double a = 0, r = 0;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) {
    const double* pp = partials + ((size_t)c * ntiles + t) * kMaxBlocksPerChannel * 2;
    a += pp[2 * b];
    r += pp[2 * b + 1];
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = r;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) {
      s0[threadIdx.x] += s0[threadIdx.x + k];
      s1[threadIdx.x] += s1[threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double zn = sqrt(s0[0]);
    const double eps = blk_eps[(size_t)ch * kMaxBlocksPerChannel + b];
    // v2 = z (1 - min(eps/||z||, 1))  (update_dual_data_fidelity.m:83)
    const double sc = zn > 0 ? 1.0 - fmin(eps / zn, 1.0) : 0.0;
    blk_scale[(size_t)ch * kMaxBlocksPerChannel + b] = (float)sc;
    const int gb = ch_blkoff[ch] + b;
    blk_stats[2 * gb] = s0[0];
    blk_stats[2 * gb + 1] = s1[0];
  }
}

int grid_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 16);
}

}  // namespace

// ------------------------------------------------------------- host side
OpView MeasOp::view() const {
  OpView v;
  const int nt = kPolyDegree + 1;
  for (int j = 0; j < kMaxTaps; ++j)
    for (int part = 0; part < 2; ++part)
      for (int k = 0; k < nt; ++k) {
        v.py[j][part][k] = j < Jy ? (float)ay.poly[((size_t)j * 2 + part) * nt + k] : 0.f;
        v.px[j][part][k] = j < Jx ? (float)ax.poly[((size_t)j * 2 + part) * nt + k] : 0.f;
      }
  v.Ny = Ny;
  v.Nx = Nx;
  v.Ky = Ky;
  v.Kx = Kx;
  v.Jy = Jy;
  v.Jx = Jx;
  v.nT0 = nT0;
  v.nT1 = nT1;
  v.nsb0 = nsb0;
  v.nsb1 = nsb1;
  v.nkeys = nkeys;
  v.tab_y = tab_y.p;
  v.tab_x = tab_x.p;
  v.sy = sy.p;
  v.sx = sx.p;
  v.geom = geom.p;
  v.sb_off = sb_off.p;
  v.ch_voff = ch_voff.p;
  v.ch_M = ch_M.p;
  return v;
}

MeasOp::~MeasOp() {
  DeviceGuard g(device);
  if (plan_all) cufftDestroy(plan_all);
  if (plan_one) cufftDestroy(plan_one);
  if (stream) cudaStreamDestroy(stream);
}

MeasOp* measop_create(int device, int Ny, int Nx, int oy, int ox, int Jy, int Jx, int L) {
  FHS_CHECK(Ny > 0 && Nx > 0 && L > 0 && oy > 0 && ox > 0, FHS_ERR_INVALID_ARG, "sizes must be positive");
  FHS_CHECK(Ny % 2 == 0 && Nx % 2 == 0, FHS_ERR_UNSUPPORTED, "Ny and Nx must be even");
  FHS_CHECK(Jy == Jx && Jy == 7, FHS_ERR_UNSUPPORTED, "this build supports 7x7 interpolation kernels");
  const int Ky = oy * Ny, Kx = ox * Nx;
  FHS_CHECK(Ky % kBinCells == 0 && Kx % kBinCells == 0, FHS_ERR_UNSUPPORTED,
            "oversampled grid sizes must be multiples of 8");
  FHS_CHECK(Ky <= 16384 && Kx <= 16384, FHS_ERR_UNSUPPORTED, "oversampled grid larger than 16384");
  FHS_CHECK(Ky >= Ny && Kx >= Nx, FHS_ERR_INVALID_ARG, "oversampling must be >= 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw Error(FHS_ERR_NO_DEVICE, "no CUDA device available");
  FHS_CHECK(device >= 0 && device < ndev, FHS_ERR_INVALID_ARG, "bad device index");
  DeviceGuard g(device);
  auto* op = new MeasOp();
  op->device = device;
  op->Ny = Ny;
  op->Nx = Nx;
  op->Ky = Ky;
  op->Kx = Kx;
  op->Jy = Jy;
  op->Jx = Jx;
  op->L = L;
  op->nsb0 = Ky / kBinCells;
  op->nsb1 = Kx / kBinCells;
  op->nT0 = ceil_div(Ky, kTileCells);
  op->nT1 = ceil_div(Kx, kTileCells);
  op->nkeys = op->nT0 * op->nT1 * kSubPerTile * kSubPerTile;
  op->ch.resize(L);
  try {
    FHS_CUDA(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking));
    op->ay = build_minmax_axis(Ny, Ky, Jy, kTableSamples);
    op->ax = (Ny == Nx && Ky == Kx) ? op->ay : build_minmax_axis(Nx, Kx, Jx, kTableSamples);
  } catch (const Error&) {
    delete op;
    throw;
  } catch (const std::exception& e) {
    delete op;
    throw Error(FHS_ERR_INVALID_ARG, e.what());
  }
  return op;
}

void measop_set_channel(MeasOp* op, int c, int64_t n, const double* om_y, const double* om_x, const double* w,
                        int n_blocks, const int64_t* block_sizes) {
  FHS_CHECK(!op->committed, FHS_ERR_STATE, "operator already committed");
  FHS_CHECK(c >= 0 && c < op->L, FHS_ERR_INVALID_ARG, "bad channel index");
  FHS_CHECK(n >= 0 && n < (int64_t)1 << 31, FHS_ERR_UNSUPPORTED, "visibilities per channel must be < 2^31");
  FHS_CHECK(n == 0 || (om_y && om_x), FHS_ERR_INVALID_ARG, "null frequency pointer");
  FHS_CHECK(n_blocks >= 1 && n_blocks <= kMaxBlocksPerChannel, FHS_ERR_UNSUPPORTED,
            "blocks per channel must be in [1, 16]");
  FHS_CHECK(block_sizes != nullptr, FHS_ERR_INVALID_ARG, "null block sizes");
  int64_t tot = 0;
  for (int b = 0; b < n_blocks; ++b) {
    FHS_CHECK(block_sizes[b] >= 0, FHS_ERR_INVALID_ARG, "negative block size");
    tot += block_sizes[b];
  }
  FHS_CHECK(tot == n, FHS_ERR_INVALID_ARG, "block sizes do not sum to n_vis");
  ChannelHost& h = op->ch[c];
  h.M = n;
  h.block_sizes.assign(block_sizes, block_sizes + n_blocks);
  // per-visibility geometry (FP64 -> offsets) and counting sort by sub-bin
  const double gy = 2.0 * M_PI / op->Ky, gx = 2.0 * M_PI / op->Kx;
  std::vector<int32_t> key(n);
  std::vector<float4> g(n);
  int blk = 0;
  int64_t blk_end = block_sizes[0];
  for (int64_t m = 0; m < n; ++m) {
    while (m >= blk_end) blk_end += block_sizes[++blk];
    FHS_CHECK(std::isfinite(om_y[m]) && std::isfinite(om_x[m]), FHS_ERR_NUMERIC, "non-finite frequency");
    const double uy = om_y[m] / gy - op->Jy / 2.0;
    const double ux = om_x[m] / gx - op->Jx / 2.0;
    const double fy0 = std::floor(uy), fx0 = std::floor(ux);
    float fy = (float)(uy - fy0), fx = (float)(ux - fx0);
    if (fy >= 1.f) fy = std::nextafter(1.f, 0.f);
    if (fx >= 1.f) fx = std::nextafter(1.f, 0.f);
    int64_t s0 = ((int64_t)fy0 + 1) % op->Ky;
    if (s0 < 0) s0 += op->Ky;
    int64_t s1 = ((int64_t)fx0 + 1) % op->Kx;
    if (s1 < 0) s1 += op->Kx;
    const unsigned kp = (unsigned)s0 | ((unsigned)s1 << 14) | ((unsigned)blk << 28);
    const float wt = w ? (float)w[m] : 1.f;
    float kpf;
    std::memcpy(&kpf, &kp, sizeof(kpf));
    g[m] = make_float4(fy, fx, kpf, wt);
    const int sb0 = (int)s0 / kBinCells, sb1 = (int)s1 / kBinCells;
    key[m] = ((sb1 / kSubPerTile) * op->nT0 + sb0 / kSubPerTile) * (kSubPerTile * kSubPerTile) +
             (sb1 % kSubPerTile) * kSubPerTile + (sb0 % kSubPerTile);
  }
  h.sb_off.assign(op->nkeys + 1, 0);
  for (int64_t m = 0; m < n; ++m) h.sb_off[key[m] + 1]++;
  for (int k = 0; k < op->nkeys; ++k) h.sb_off[k + 1] += h.sb_off[k];
  std::vector<int32_t> pos(h.sb_off.begin(), h.sb_off.end() - 1);
  h.geom.resize(n);
  h.perm.resize(n);
  for (int64_t m = 0; m < n; ++m) {
    const int32_t p = pos[key[m]]++;
    h.geom[p] = g[m];
    h.perm[p] = (int32_t)m;
  }
  h.set = true;
}

void measop_commit(MeasOp* op) {
  FHS_CHECK(!op->committed, FHS_ERR_STATE, "operator already committed");
  for (int c = 0; c < op->L; ++c) FHS_CHECK(op->ch[c].set, FHS_ERR_STATE, "channel " + std::to_string(c) + " not set");
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  const int L = op->L;
  op->h_voff.resize(L);
  op->h_M.resize(L);
  op->h_blkoff.resize(L);
  op->h_nblk.resize(L);
  int64_t vo = 0;
  int bo = 0;
  op->maxM = 0;
  for (int c = 0; c < L; ++c) {
    op->h_voff[c] = vo;
    op->h_M[c] = (int32_t)op->ch[c].M;
    op->h_blkoff[c] = bo;
    op->h_nblk[c] = (int32_t)op->ch[c].block_sizes.size();
    vo += op->ch[c].M;
    bo += op->h_nblk[c];
    op->maxM = std::max(op->maxM, op->ch[c].M);
  }
  op->Mtot = vo;
  op->nblk_tot = bo;
  // tables and scaling factors (FP32 copies of the FP64 construction)
  auto upload_table = [&](const MinMaxAxis& a, DevBuf<float2>& t, DevBuf<float>& sc) {
    std::vector<float2> h((size_t)a.J * (kTableSamples + 1));
    for (size_t i = 0; i < h.size(); ++i) h[i] = make_float2((float)a.table_re[i], (float)a.table_im[i]);
    t.alloc(h.size());
    t.upload(h.data(), h.size(), s);
    std::vector<float> hs(a.scale.begin(), a.scale.end());
    sc.alloc(hs.size());
    sc.upload(hs.data(), hs.size(), s);
  };
  upload_table(op->ay, op->tab_y, op->sy);
  upload_table(op->ax, op->tab_x, op->sx);
  op->geom.alloc(std::max<int64_t>(op->Mtot, 1));
  op->zbuf.alloc(std::max<int64_t>(op->Mtot, 1));
  op->perm.alloc(std::max<int64_t>(op->Mtot, 1));
  op->sb_off.alloc((size_t)L * (op->nkeys + 1));
  for (int c = 0; c < L; ++c) {
    const ChannelHost& h = op->ch[c];
    if (h.M) {
      FHS_CUDA(cudaMemcpyAsync(op->geom.p + op->h_voff[c], h.geom.data(), h.M * sizeof(float4),
                               cudaMemcpyHostToDevice, s));
      FHS_CUDA(cudaMemcpyAsync(op->perm.p + op->h_voff[c], h.perm.data(), h.M * sizeof(int32_t),
                               cudaMemcpyHostToDevice, s));
    }
    FHS_CUDA(cudaMemcpyAsync(op->sb_off.p + (size_t)c * (op->nkeys + 1), h.sb_off.data(),
                             (op->nkeys + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  }
  op->ch_voff.alloc(L);
  op->ch_voff.upload(op->h_voff.data(), L, s);
  op->ch_M.alloc(L);
  op->ch_M.upload(op->h_M.data(), L, s);
  op->ch_blkoff.alloc(L);
  op->ch_blkoff.upload(op->h_blkoff.data(), L, s);
  op->ch_nblk.alloc(L);
  op->ch_nblk.upload(op->h_nblk.data(), L, s);
  const size_t gsz = (size_t)L * op->No();
  op->pad.alloc(gsz);
  op->pad.zero(s);
  op->gridA.alloc(gsz);
  op->gridB.alloc(gsz);
  op->gridB.zero(s);
  op->partials.alloc((size_t)L * op->ntiles() * kMaxBlocksPerChannel * 2);
  op->blk_stats.alloc((size_t)std::max(op->nblk_tot, 1) * 2);
  op->blk_scale.alloc((size_t)L * kMaxBlocksPerChannel);
  op->blk_scale.zero(s);
  op->blk_eps.alloc((size_t)L * kMaxBlocksPerChannel);
  op->blk_eps.zero(s);
  int n[2] = {op->Kx, op->Ky};
  FHS_CUFFT(cufftPlanMany(&op->plan_all, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, L));
  FHS_CUFFT(cufftSetStream(op->plan_all, s));
  FHS_CUFFT(cufftPlanMany(&op->plan_one, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, 1));
  FHS_CUFFT(cufftSetStream(op->plan_one, s));
  FHS_CUDA(cudaStreamSynchronize(s));
  // host copies of the sorted geometry are no longer needed
  for (auto& h : op->ch) {
    std::vector<float4>().swap(h.geom);
    std::vector<int32_t>().swap(h.perm);
  }
  op->committed = true;
}

void launch_pad(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s) {
  dim3 grid(grid_blocks(op->Npix(), 256), np);
  pad_kernel<<<grid, 256, 0, s>>>(x, op->pad.p, op->sy.p, op->sx.p, op->Ny, op->Nx, op->Ky, op->Kx, p0);
  count_launch();
  FHS_LAUNCH_CHECK();
}

static void fft_exec(const MeasOp* op, float2* in, float2* out, int p0, int np, int dir) {
  const size_t No = op->No();
  if (np == op->L && p0 == 0) {
    FHS_CUFFT(cufftExecC2C(op->plan_all, (cufftComplex*)in, (cufftComplex*)out, dir));
  } else {
    for (int p = p0; p < p0 + np; ++p)
      FHS_CUFFT(cufftExecC2C(op->plan_one, (cufftComplex*)(in + p * No), (cufftComplex*)(out + p * No), dir));
  }
}

void fft_forward(const MeasOp* op, int p0, int np, cudaStream_t s) {
  (void)s;
  fft_exec(op, op->pad.p, op->gridA.p, p0, np, CUFFT_FORWARD);
}

void fft_inverse(const MeasOp* op, int p0, int np, cudaStream_t s) {
  (void)s;
  fft_exec(op, op->gridB.p, op->gridA.p, p0, np, CUFFT_INVERSE);
}

void launch_degrid_plain(const MeasOp* op, int c0, int nc, float2* out, cudaStream_t s) {
  dim3 grid(op->ntiles(), nc);
  degrid_kernel<7, false><<<grid, 256, 0, s>>>(op->view(), op->gridA.p, c0, out, nullptr, nullptr, nullptr,
                                               nullptr, nullptr);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_grid_plain(const MeasOp* op, int c0, int nc, const float2* v, cudaStream_t s) {
  dim3 grid(op->ntiles(), nc);
  grid_kernel<7, false><<<grid, 256, 0, s>>>(op->view(), op->gridB.p, c0, v, nullptr, nullptr, nullptr);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_crop_real(const MeasOp* op, float* out, const float* sigma, int p0, int np, cudaStream_t s) {
  dim3 grid(grid_blocks(op->Npix(), 256), np);
  crop_real_kernel<<<grid, 256, 0, s>>>(op->gridA.p, out, sigma, op->sy.p, op->sx.p, op->Ny, op->Nx, op->Ky,
                                        op->Kx, p0);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_degrid_dual(const MeasOp* op, int c0, int nc, float2* v2, float2* gold, const float2* y,
                        cudaStream_t s) {
  dim3 grid(op->ntiles(), nc);
  degrid_kernel<7, true><<<grid, 256, 0, s>>>(op->view(), op->gridA.p, c0, nullptr, v2, gold, y,
                                              op->partials.p, op->zbuf.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_block_reduce(const MeasOp* op, int c0, int nc, cudaStream_t s) {
  dim3 grid(nc, kMaxBlocksPerChannel);
  block_reduce_kernel<<<grid, 256, 0, s>>>(op->partials.p, op->ntiles(), c0, op->ch_nblk.p, op->ch_blkoff.p,
                                           op->blk_eps.p, op->blk_scale.p, op->blk_stats.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_grid_dual(const MeasOp* op, int c0, int nc, float2* v2, cudaStream_t s) {
  dim3 grid(op->ntiles(), nc);
  grid_kernel<7, true><<<grid, 256, 0, s>>>(op->view(), op->gridB.p, c0, nullptr, v2, op->blk_scale.p,
                                            op->zbuf.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
