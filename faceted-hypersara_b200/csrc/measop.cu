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
// in the tile.  Gridding: one CTA per tile accumulates, in warp-private
// shared-memory bands, the taps of the visibilities that start in the tile
// or in the 8-cell ring below it, then writes the tile once: no atomics of
// any kind, no grid zeroing.
#include "measop.cuh"
#include "cplx.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace fhs {

unsigned long long g_launches = 0;

namespace {

constexpr int kSmemPitch = kTileCells + kBinCells;  // 72 (>= 64 + J - 1)

// ---------------------------------------------------------------- degrid
// MODE 0: out = G Fx.  MODE 1: l2-ball dual, pass 1.  MODE 2: ellipsoid dual,
// pass 1 (d = v2/pU + 2 GFx - gold - y to zbuf, block norms of the first FB
// point t_1 - y = w0 + (mu/pU)(d - w0), w0 = proj - y).
// NB: blocks per channel the per-thread FP64 norm accumulators cover (dual
// modes; shared-memory FP64 atomics per visibility would serialise the warp).
// HALF: the grid is the half spectrum of a real-to-complex FFT,
// [Kx][Ky/2 + 1] per channel; G(k0, k1) for k0 > Ky/2 is conj(G(-k0, -k1)).
template <int J, int MODE, int NB, bool HALF>
__global__ void __launch_bounds__(256, 3) degrid_kernel(OpView op, const float2* __restrict__ grid,
                                                     const WorkItem* __restrict__ items,
                                                     const int* __restrict__ order, int item0,
                                                     float2* __restrict__ out, const float2* __restrict__ v2,
                                                     float2* __restrict__ gold,
                                                     const float2* __restrict__ y,
                                                     double* __restrict__ partials, float2* __restrict__ zbuf,
                                                     PrecondView pc) {
  constexpr bool DUAL = MODE != 0;
  // pitch 72 along y: starts within a sub-bin spread over distinct bank pairs
  constexpr int P = kSmemPitch;
  constexpr int R = kTileCells + J - 1;
  __shared__ float2 sm[R * P];
  __shared__ float2 psy[R], psx[R];   // cell phases psi of the staged rows / columns
  __shared__ double bacc[kMaxBlocksPerChannel * 2];
  const WorkItem it = items[order ? order[blockIdx.x] : item0 + blockIdx.x];
  const int tile = it.tile;
  const int ch = it.ch;
  const int t0 = tile % op.nT0, t1 = tile / op.nT0;
  const int32_t* off = op.sb_off + (size_t)ch * (op.nkeys + 1);
  const int tb = off[tile * kSubPerTile * kSubPerTile];
  const int te = off[(tile + 1) * kSubPerTile * kSubPerTile];
  const int beg = tb + (int)(((int64_t)(te - tb) * it.split) / it.nsplit);
  const int end = tb + (int)(((int64_t)(te - tb) * (it.split + 1)) / it.nsplit);
  if (DUAL) {
    if (threadIdx.x < kMaxBlocksPerChannel * 2) bacc[threadIdx.x] = 0.0;
  }
  const int a0 = t0 * kTileCells, a1 = t1 * kTileCells;
  const int Kh = op.Ky / 2 + 1;
  const float2* g = grid + (size_t)ch * (HALF ? Kh : op.Ky) * op.Kx;
  if (threadIdx.x < R) {
    psy[threadIdx.x] = cell_phase(wrap(a0 + threadIdx.x, op.Ky), op.Ky);
  } else if (threadIdx.x >= 128 && threadIdx.x < 128 + R) {
    psx[threadIdx.x - 128] = cell_phase(wrap(a1 + threadIdx.x - 128, op.Kx), op.Kx);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < R * R; idx += blockDim.x) {
    const int c1 = idx / R, cc0 = idx - c1 * R;
    const int k0 = wrap(a0 + cc0, op.Ky), k1 = wrap(a1 + c1, op.Kx);
    float2 gv;
    if (!HALF) {
      gv = __ldg(g + (size_t)k1 * op.Ky + k0);
    } else if (k0 < Kh) {
      gv = __ldg(g + (size_t)k1 * Kh + k0);
    } else {  // Hermitian mirror
      const float2 m = __ldg(g + (size_t)(k1 == 0 ? 0 : op.Kx - k1) * Kh + (op.Ky - k0));
      gv = make_float2(m.x, -m.y);
    }
    sm[c1 * P + cc0] = cmul(cmul(psy[cc0], psx[c1]), gv);   // psi_y psi_x G
  }
  __syncthreads();
  double nacc[NB][2];
#pragma unroll
  for (int b = 0; b < NB; ++b) nacc[b][0] = nacc[b][1] = 0.0;
  const int64_t vo = op.ch_voff[ch];
  // software pipeline: the next visibility's geometry and dual operands are
  // loaded while this one is interpolated
  float4 gm_n = make_float4(0.f, 0.f, 0.f, 0.f);
  float2 yv_n = make_float2(0.f, 0.f), vv_n = yv_n, go_n = yv_n, ph_n = yv_n;
  auto fetch = [&](int i) {
    gm_n = __ldg(op.geom + vo + i);
    ph_n = __ldg(op.vph + vo + i);
    if (DUAL) {
      yv_n = y[vo + i];
      vv_n = v2[vo + i];
      go_n = gold[vo + i];
    }
  };
  if (beg + (int)threadIdx.x < end) fetch(beg + threadIdx.x);
  for (int i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const float4 gm = gm_n;
    const float2 yv = yv_n, vv = vv_n, go = go_n, ph = ph_n;
    if (i + (int)blockDim.x < end) fetch(i + blockDim.x);
    const unsigned kp = __float_as_uint(gm.z);
    const int s0 = (int)(kp & 0x3FFFu), s1 = (int)((kp >> 14) & 0x3FFFu);
    const int d0 = s0 - a0, d1 = s1 - a1;
    float fy, fx;
    int ksy, ksx;
    axis_start(gm.x, s0, op.Ky, fy, ksy);
    axis_start(gm.y, s1, op.Kx, fx, ksx);
    float cy[J], cx[J];
    rtaps<J>(op.ry, fy, cy);
    rtaps<J>(op.rx, fx, cx);
    tap_signs<J>(ksy, op.Ky, cy);
    tap_signs<J>(ksx, op.Kx, cx);
    // real taps on the phase-multiplied tile: two FMAs per tap and column
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int jx = 0; jx < J; ++jx) {
      const float2* col = sm + (d1 + jx) * P + d0;
      float2 sc = make_float2(0.f, 0.f);
#pragma unroll
      for (int jy = 0; jy < J; ++jy) {
        const float2 gv = col[jy];
        sc.x = fmaf(cy[jy], gv.x, sc.x);
        sc.y = fmaf(cy[jy], gv.y, sc.y);
      }
      acc.x = fmaf(cx[jx], sc.x, acc.x);
      acc.y = fmaf(cx[jx], sc.y, acc.y);
    }
    const float2 pa = cmul(ph, acc);
    const float2 gfx = make_float2(gm.w * pa.x, gm.w * pa.y);
    if (!DUAL) {
      out[vo + i] = gfx;
    } else {
      const float2 r = make_float2(gfx.x - yv.x, gfx.y - yv.y);
      const int blk = (int)(kp >> 28);
      double n0;
      if (MODE == 1) {
        const float2 z = make_float2(vv.x + 2.f * gfx.x - go.x - yv.x, vv.y + 2.f * gfx.y - go.y - yv.y);
        zbuf[vo + i] = z;
        n0 = (double)z.x * z.x + (double)z.y * z.y;
      } else {
        const float ip = 1.f / pc.pu[vo + i];
        const float2 d = make_float2(fmaf(vv.x, ip, 2.f * gfx.x - go.x - yv.x),
                                     fmaf(vv.y, ip, 2.f * gfx.y - go.y - yv.y));
        zbuf[vo + i] = d;
        const double2 w0 = pc.w[vo + i];
        const double m = (double)pc.mu[(size_t)ch * kMaxBlocksPerChannel + blk] * (double)ip;
        const double tx = fma(m, (double)d.x - w0.x, w0.x), ty = fma(m, (double)d.y - w0.y, w0.y);
        n0 = tx * tx + ty * ty;
      }
      gold[vo + i] = gfx;
      const double n1 = (double)r.x * r.x + (double)r.y * r.y;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        if (b == blk) {
          nacc[b][0] += n0;
          nacc[b][1] += n1;
        }
      }
    }
  }
  if (DUAL) {
    // warp sums, then one shared atomic per warp and value
#pragma unroll
    for (int b = 0; b < NB; ++b) {
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        double v = nacc[b][f];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&bacc[2 * b + f], v);
      }
    }
    __syncthreads();
    if (threadIdx.x < kMaxBlocksPerChannel * 2)
      partials[(size_t)it.slot * kMaxBlocksPerChannel * 2 + threadIdx.x] = bacc[threadIdx.x];
  }
}

// ------------------------------------------------------------------ grid
// One CTA (8 warps) per 64x64 grid tile and channel, or per slice of a very
// dense tile.  The tile's accumulator is FP32 complex in shared memory with
// an even column pitch of 66 (16-byte aligned row pairs; the quarter-warp
// accesses of a patch column fall on distinct bank groups).  Visibilities
// that start in the tile or in the 8-cell ring above / left of it reach the
// tile; taps that fall outside it are dropped (the neighbouring tile adds
// them through its own ring).
//
// The 81 sub-bins that feed the tile (8x8 own + the ring) are processed in
// four phases by the parity of their sub-bin row and column: two sub-bins of
// one phase are 16 cells apart and the taps of a sub-bin's visibilities
// cover 8 + 6 = 14 cells, so within a phase no two sub-bins touch the same
// accumulator cell.  Warps claim the phase's sub-bins dynamically, largest
// first (the per-item schedule is built on the host, GridPlan), and own them
// outright: no atomics, no per-warp copies of the tile, and a fixed
// summation order per cell (deterministic results).  Five warps per CTA fit
// the phase sizes of a full tile (25, 20, 20, 16 sub-bins) in whole rounds.
//
// Inside a sub-bin the visibilities are visited grouped by 2x2 block of
// start cells (gperm: block-major order).  All visibilities of a block touch
// the same 8x8 patch, which the warp holds in registers (lane: column
// lane & 7, rows 2 (lane >> 3) + {0, 1}).  The taps are phase-factored
// (cplx.cuh): the patch accumulates real row taps sigma c_y (8 rows, zero
// padded) times conj(phase) w v sigma c_x (8 columns), two real-by-complex
// FMAs per lane and visibility; the cell phases conj(psi_y psi_x) are
// applied once per cell when the tile is written.  A patch is added into the
// shared accumulator once per block, and the tile is written once.
constexpr int kGPitch = kTileCells + 2;             // 66
constexpr int kGWarps = 5;
constexpr int kGStage = 28;                         // floats per staged visibility: 8 a + 8 complex b + 4 pad
constexpr int kGSub = (kSubPerTile + 1) * (kSubPerTile + 1);  // 81 sub-bins feed a tile

// adds a lane's two patch cells (rows row, row + 1 of column col, tile
// coordinates) into the accumulator; cells outside the tile are dropped
static __device__ __forceinline__ void patch_flush(float2* acc, int row, int col, float2 p0, float2 p1) {
  if (row >= 0 && row < kTileCells && col >= 0 && col < kTileCells) {
    float4* cell = reinterpret_cast<float4*>(acc + col * kGPitch + row);
    float4 c = *cell;
    c.x += p0.x;
    c.y += p0.y;
    c.z += p1.x;
    c.w += p1.y;
    *cell = c;
  }
}

// MODE 0: gridB = G^H vin.  MODE 1: l2-ball dual, pass 2 (v2 = z scale).
// MODE 2: ellipsoid dual, pass 2 (v2 = pU (d - w), w = proj - y).
template <int J, int MODE>
__global__ void __launch_bounds__(kGWarps * 32, 4) grid_kernel(OpView op, float2* __restrict__ gridB,
                                                               const WorkItem* __restrict__ items,
                                                               const int* __restrict__ order, int item0,
                                                               float2* __restrict__ partial,
                                                               const float2* __restrict__ vin,
                                                               float2* __restrict__ v2,
                                                               const float* __restrict__ blk_scale,
                                                               const float2* __restrict__ zbuf, PrecondView pc,
                                                               const int32_t* __restrict__ gperm,
                                                               const GridPlan* __restrict__ plans) {
  static_assert(J == 7, "the 8x8 patch of a 2x2 start block holds 7 taps per axis");
  constexpr bool DUAL = MODE != 0;
  extern __shared__ float4 gsm4[];
  float2* acc = reinterpret_cast<float2*>(gsm4);                 // [kTileCells cols][kGPitch]
  float* stage_all = reinterpret_cast<float*>(acc + kTileCells * kGPitch);   // [warps][32][kGStage]
  __shared__ float2 psy[kTileCells], psx[kTileCells];             // cell phases of the tile's rows / columns
  __shared__ int2 rng[kGSub];
  __shared__ GridPlan plan;
  __shared__ int pclaim[4];
  const int itx = order ? order[blockIdx.x] : item0 + blockIdx.x;
  const WorkItem it = items[itx];
  const int tile = it.tile;
  const int ch = it.ch;
  const int t0 = tile % op.nT0, t1 = tile / op.nT0;
  const int a0 = t0 * kTileCells, a1 = t1 * kTileCells;
  const int T0 = min(kTileCells, op.Ky - a0), T1 = min(kTileCells, op.Kx - a1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t* off = op.sb_off + (size_t)ch * (op.nkeys + 1);
  if (threadIdx.x < (int)(sizeof(GridPlan) / 4))
    reinterpret_cast<int*>(&plan)[threadIdx.x] = reinterpret_cast<const int*>(plans + itx)[threadIdx.x];
  if (threadIdx.x < 4) pclaim[threadIdx.x] = 0;
  if (threadIdx.x >= 32 && threadIdx.x < 32 + kTileCells) {
    const int r = threadIdx.x - 32;
    psy[r] = cell_phase(wrap(a0 + r, op.Ky), op.Ky);
    psx[r] = cell_phase(wrap(a1 + r, op.Kx), op.Kx);
  }
  // ---- the 81 sub-bins: (i, j) in [-1, 8)^2, -1 = the ring (wraps)
  if (threadIdx.x >= 64 && threadIdx.x < 64 + kGSub) {
    const int t = threadIdx.x - 64;
    const int i = t % (kSubPerTile + 1) - 1, j = t / (kSubPerTile + 1) - 1;
    const int nrows = min(kSubPerTile, op.nsb0 - t0 * kSubPerTile);
    const int ncols = min(kSubPerTile, op.nsb1 - t1 * kSubPerTile);
    int2 r = make_int2(0, 0);
    if (i < nrows && j < ncols) {
      const int sb0 = i < 0 ? (t0 * kSubPerTile - 1 + op.nsb0) % op.nsb0 : t0 * kSubPerTile + i;
      const int sb1 = j < 0 ? (t1 * kSubPerTile - 1 + op.nsb1) % op.nsb1 : t1 * kSubPerTile + j;
      const int key = ((sb1 / kSubPerTile) * op.nT0 + sb0 / kSubPerTile) * (kSubPerTile * kSubPerTile) +
                      (sb1 % kSubPerTile) * kSubPerTile + (sb0 % kSubPerTile);
      const int b = off[key], e = off[key + 1];
      const int len = e - b;
      r.x = b + (int)(((int64_t)len * it.split) / it.nsplit);
      r.y = b + (int)(((int64_t)len * (it.split + 1)) / it.nsplit);
    }
    rng[t] = r;
  }
  __syncthreads();
  // split tiles write a partial tile (summed by grid_combine_kernel)
  float2* gb;
  size_t ld;
  int g0, g1;
  if (it.slot >= 0) {
    gb = partial + (size_t)it.slot * kTileCells * kTileCells;
    ld = kTileCells;
    g0 = 0;
    g1 = 0;
  } else {
    gb = gridB + (size_t)ch * op.Ky * op.Kx;
    ld = op.Ky;
    g0 = a0;
    g1 = a1;
  }
  const int nsub = plan.count[0] + plan.count[1] + plan.count[2] + plan.count[3];
  if (nsub == 0) {   // nothing reaches the tile: zeros
    for (int idx = threadIdx.x; idx < T0 * T1; idx += blockDim.x) {
      const int cc1 = idx / T0, cc0 = idx - cc1 * T0;
      gb[(size_t)(g1 + cc1) * ld + g0 + cc0] = make_float2(0.f, 0.f);
    }
    return;
  }
  for (int k = threadIdx.x; k < kTileCells * kGPitch / 2; k += blockDim.x) gsm4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  const int64_t vo = op.ch_voff[ch];
  const float* scl = DUAL ? blk_scale + (size_t)ch * kMaxBlocksPerChannel : nullptr;
  float* st = stage_all + warp * 32 * kGStage;
  const int pc_col = lane & 7, pc_rp = lane >> 3;   // this lane's patch column and row pair
  const float2* sa = reinterpret_cast<const float2*>(st + 2 * pc_rp);      // staged row taps of its two rows
  const float2* sbp = reinterpret_cast<const float2*>(st + 8 + 2 * pc_col);  // staged column value
  constexpr int kSt2 = kGStage / 2;                                         // float2 per staged visibility
  int pbase = 0;
  for (int ph = 0; ph < 4; ++ph) {
    const int nph = plan.count[ph];
    for (;;) {
      int idx = 0;
      if (lane == 0) idx = atomicAdd(&pclaim[ph], 1);
      idx = __shfl_sync(0xffffffffu, idx, 0);
      if (idx >= nph) break;
      const int sb = plan.sub[pbase + idx];
      const int2 r = rng[sb];
      const int i = sb % (kSubPerTile + 1) - 1, j = sb / (kSubPerTile + 1) - 1;
      const bool own = i >= 0 && j >= 0;
      const int rowb = kBinCells * i + 2 * pc_rp, colb = kBinCells * j + pc_col;   // tile coordinates
      float2 p0 = make_float2(0.f, 0.f), p1 = p0;   // this lane's two patch cells
      int cur = -1;                                  // 2x2 start block held in p0/p1
      for (int base = r.x; base < r.y; base += 32) {
        const int n = min(32, r.y - base);
        int blk = 16;
        if (lane < n) {
          const int q = gperm[vo + base + lane];      // channel-relative storage index
          const float4 gm = __ldg(op.geom + vo + q);
          const unsigned kp = __float_as_uint(gm.z);
          const int s0 = (int)(kp & 0x3FFFu), s1 = (int)((kp >> 14) & 0x3FFFu);
          float2 v;
          if (MODE == 1) {
            const float2 z = zbuf[vo + q];
            const float sc = scl[kp >> 28];
            v = make_float2(z.x * sc, z.y * sc);
            if (own) v2[vo + q] = v;   // the owner tile writes the dual
          } else if (MODE == 2) {
            const float2 d = zbuf[vo + q];
            const double2 w = pc.w[vo + q];
            const double pu = (double)pc.pu[vo + q];
            v = make_float2((float)(pu * ((double)d.x - w.x)), (float)(pu * ((double)d.y - w.y)));
            if (own) v2[vo + q] = v;
          } else {
            v = vin[vo + q];
          }
          float fy, fx;
          int ksy, ksx;
          axis_start(gm.x, s0, op.Ky, fy, ksy);
          axis_start(gm.y, s1, op.Kx, fx, ksx);
          float cy[J], cx[J];
          rtaps<J>(op.ry, fy, cy);
          rtaps<J>(op.rx, fx, cx);
          tap_signs<J>(ksy, op.Ky, cy);
          tap_signs<J>(ksx, op.Kx, cx);
          v = cmulc(__ldg(op.vph + vo + q), make_float2(v.x * gm.w, v.y * gm.w));   // conj(phase) w v
          // zero-padded 8-tap rows / columns of the 2x2 block's patch
          const bool dy = s0 & 1, dx = s1 & 1;
          float ap[8], bp[8];
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            ap[t] = dy ? (t > 0 ? cy[t - 1] : 0.f) : (t < J ? cy[t] : 0.f);
            bp[t] = dx ? (t > 0 ? cx[t - 1] : 0.f) : (t < J ? cx[t] : 0.f);
          }
          float4* sl = reinterpret_cast<float4*>(st + lane * kGStage);
          sl[0] = make_float4(ap[0], ap[1], ap[2], ap[3]);
          sl[1] = make_float4(ap[4], ap[5], ap[6], ap[7]);
#pragma unroll
          for (int t = 0; t < 4; ++t)
            sl[2 + t] = make_float4(bp[2 * t] * v.x, bp[2 * t] * v.y, bp[2 * t + 1] * v.x, bp[2 * t + 1] * v.y);
          blk = ((s0 & 7) >> 1) | (((s1 & 7) >> 1) << 2);
        }
        int prev = __shfl_up_sync(0xffffffffu, blk, 1);
        if (lane == 0) prev = cur;
        const unsigned change = __ballot_sync(0xffffffffu, lane < n && blk != prev);
        __syncwarp();
        int k = 0;
        while (k < n) {   // runs of one 2x2 block (warp-uniform bounds)
          if ((change >> k) & 1u) {
            if (cur >= 0) patch_flush(acc, rowb + 2 * (cur & 3), colb + 2 * (cur >> 2), p0, p1);
            cur = __shfl_sync(0xffffffffu, blk, k);
            p0 = make_float2(0.f, 0.f);
            p1 = p0;
          }
          const unsigned rest = change & ~((2u << k) - 1u);
          const int kend = rest ? __ffs(rest) - 1 : n;
          for (; k + 2 <= kend; k += 2) {
            const float2 a = sa[k * kSt2], b = sbp[k * kSt2];
            const float2 a2 = sa[(k + 1) * kSt2], b2 = sbp[(k + 1) * kSt2];
            p0.x = fmaf(a.x, b.x, p0.x);
            p0.y = fmaf(a.x, b.y, p0.y);
            p1.x = fmaf(a.y, b.x, p1.x);
            p1.y = fmaf(a.y, b.y, p1.y);
            p0.x = fmaf(a2.x, b2.x, p0.x);
            p0.y = fmaf(a2.x, b2.y, p0.y);
            p1.x = fmaf(a2.y, b2.x, p1.x);
            p1.y = fmaf(a2.y, b2.y, p1.y);
          }
          if (k < kend) {
            const float2 a = sa[k * kSt2], b = sbp[k * kSt2];
            p0.x = fmaf(a.x, b.x, p0.x);
            p0.y = fmaf(a.x, b.y, p0.y);
            p1.x = fmaf(a.y, b.x, p1.x);
            p1.y = fmaf(a.y, b.y, p1.y);
            ++k;
          }
        }
        __syncwarp();   // the stage is rewritten by the next chunk
      }
      if (cur >= 0) patch_flush(acc, rowb + 2 * (cur & 3), colb + 2 * (cur >> 2), p0, p1);
    }
    pbase += nph;
    __syncthreads();   // the next phase's sub-bins overlap this phase's patches
  }
  if (T0 == kTileCells) {
    for (int idx = threadIdx.x; idx < kTileCells * T1; idx += blockDim.x) {
      const int c = idx >> 6, rr = idx & (kTileCells - 1);
      gb[(size_t)(g1 + c) * ld + g0 + rr] = cmulc(cmul(psy[rr], psx[c]), acc[c * kGPitch + rr]);  // conj(psi) acc
    }
  } else {
    for (int idx = threadIdx.x; idx < T0 * T1; idx += blockDim.x) {
      const int c = idx / T0, rr = idx - c * T0;
      gb[(size_t)(g1 + c) * ld + g0 + rr] = cmulc(cmul(psy[rr], psx[c]), acc[c * kGPitch + rr]);
    }
  }
}

// Sums the partial tiles of split tiles into the grid (fixed order: deterministic).
__global__ void __launch_bounds__(256) grid_combine_kernel(OpView op, float2* __restrict__ gridB,
                                                           const GridCombine* __restrict__ comb,
                                                           const float2* __restrict__ partial) {
  const GridCombine c = comb[blockIdx.x];
  const int t0 = c.tile % op.nT0, t1 = c.tile / op.nT0;
  const int a0 = t0 * kTileCells, a1 = t1 * kTileCells;
  const int T0 = min(kTileCells, op.Ky - a0), T1 = min(kTileCells, op.Kx - a1);
  float2* gb = gridB + (size_t)c.ch * op.Ky * op.Kx;
  for (int idx = threadIdx.x; idx < T0 * T1; idx += blockDim.x) {
    const int cc1 = idx / T0, cc0 = idx - cc1 * T0;
    float2 v = make_float2(0.f, 0.f);
    for (int k = 0; k < c.nsplit; ++k) {
      const float2 p = partial[(size_t)(c.pbase + k) * kTileCells * kTileCells + (size_t)cc1 * kTileCells + cc0];
      v.x += p.x;
      v.y += p.y;
    }
    gb[(size_t)(a1 + cc1) * op.Ky + a0 + cc0] = v;
  }
}

constexpr size_t kGridSmem = (size_t)kTileCells * kGPitch * sizeof(float2) +
                             (size_t)kGWarps * 32 * kGStage * sizeof(float);

template <int J, int MODE>
void launch_grid_kernel(const MeasOp* op, int c0, int nc, const float2* vin, float2* v2, const float* scale,
                        const float2* zbuf, PrecondView pc, cudaStream_t s) {
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(grid_kernel<J, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGridSmem));
    attr[dev] = true;
  }
  const int i0 = op->h_gr_off[c0], n = op->h_gr_off[c0 + nc] - i0;
  if (n > 0) {
    // the whole operator at once: items largest first (gr_order), so the
    // densest tiles do not end up in the tail of the launch
    const bool all = c0 == 0 && nc == op->L;
    grid_kernel<J, MODE><<<n, kGWarps * 32, kGridSmem, s>>>(op->view(), op->gridB.p, op->gr_items.p,
                                                            all ? op->gr_order.p : nullptr, i0,
                                                            op->gr_partial.p, vin, v2, scale, zbuf, pc,
                                                            op->gperm.p, op->gr_plan.p);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
  const int k0 = op->h_comb_off[c0], nk = op->h_comb_off[c0 + nc] - k0;
  if (nk > 0) {
    grid_combine_kernel<<<nk, 256, 0, s>>>(op->view(), op->gridB.p, op->gr_combine.p + k0, op->gr_partial.p);
    count_launch();
    FHS_LAUNCH_CHECK();
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

__global__ void block_reduce_kernel(const double* __restrict__ partials, const int* __restrict__ slot_off, int c0,
                                    const int32_t* __restrict__ ch_nblk, const int32_t* __restrict__ ch_blkoff,
                                    const double* __restrict__ blk_eps, float* __restrict__ blk_scale,
                                    double* __restrict__ blk_stats, int mode, double* __restrict__ fb_c,
                                    int* __restrict__ fb_iter) {
  const int ch = c0 + blockIdx.x;
  const int b = blockIdx.y;
  if (b >= ch_nblk[ch]) return;
  __shared__ double s0[256], s1[256];
  double a = 0, r = 0;
  for (int t = slot_off[ch] + threadIdx.x; t < slot_off[ch + 1]; t += blockDim.x) {
    const double* pp = partials + (size_t)t * kMaxBlocksPerChannel * 2;
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
    const size_t k = (size_t)ch * kMaxBlocksPerChannel + b;
    const double eps = blk_eps[k];
    if (mode == 0) {
      // v2 = z (1 - min(eps/||z||, 1))  (update_dual_data_fidelity.m:83)
      const double sc = zn > 0 ? 1.0 - fmin(eps / zn, 1.0) : 0.0;
      blk_scale[k] = (float)sc;
    } else {
      // first FB point of the ellipsoid projection: scale of P_B(t_1)
      fb_c[k] = zn > eps ? eps / zn : 1.0;
      fb_iter[k] = 0;
    }
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
  for (int j = 0; j < kMaxTaps; ++j)
    for (int k = 0; k < nt; ++k) {
      v.ry[j][k] = j < Jy ? (float)ay.poly_real[(size_t)j * nt + k] : 0.f;
      v.rx[j][k] = j < Jx ? (float)ax.poly_real[(size_t)j * nt + k] : 0.f;
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
  v.vph = vph.p;
  v.sb_off = sb_off.p;
  v.ch_voff = ch_voff.p;
  v.ch_M = ch_M.p;
  return v;
}

MeasOp::~MeasOp() {
  DeviceGuard g(device);
  if (plan_all) cufftDestroy(plan_all);
  if (plan_one) cufftDestroy(plan_one);
  if (plan_r2c) cufftDestroy(plan_r2c);
  if (plan_c2r) cufftDestroy(plan_c2r);
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
    // frequencies are 2 pi periodic (integer pixel positions): take them in [-pi, pi)
    const double oyn = om_y[m] - 2.0 * M_PI * std::floor((om_y[m] + M_PI) / (2.0 * M_PI));
    const double oxn = om_x[m] - 2.0 * M_PI * std::floor((om_x[m] + M_PI) / (2.0 * M_PI));
    const double uy = oyn / gy - op->Jy / 2.0;
    const double ux = oxn / gx - op->Jx / 2.0;
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
    // the sign bit of the fractional offsets marks a negative unwrapped
    // first tap k0 + 1 (the kernels resolve the grid wrap with it)
    if (fy0 + 1 < 0) fy = std::copysign(fy, -1.f);
    if (fx0 + 1 < 0) fx = std::copysign(fx, -1.f);
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
  // Inside each sub-bin, deal the visibilities round-robin over the 16
  // classes (start row mod 8, start column mod 2): the degridding threads of a
  // half-warp then read their taps' grid values (float2, column pitch 72) from
  // 16 distinct bank pairs in the dense sub-bins.
  std::vector<float4> tg;
  std::vector<int32_t> tp, order;
  for (int k = 0; k < op->nkeys; ++k) {
    const int a = h.sb_off[k], b = h.sb_off[k + 1];
    if (b - a < 2) continue;
    int cnt[16] = {0};
    order.assign(b - a, 0);
    for (int i = a; i < b; ++i) {
      unsigned kp;
      std::memcpy(&kp, &h.geom[i].z, sizeof(kp));
      const int c = (int)(kp & 7u) + 8 * (int)((kp >> 14) & 1u);
      order[i - a] = cnt[c]++ * 16 + c;  // (rank within its class, class)
    }
    std::vector<int32_t> idx(b - a);
    for (int i = 0; i < b - a; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int u, int v) { return order[u] < order[v]; });
    tg.assign(h.geom.begin() + a, h.geom.begin() + b);
    tp.assign(h.perm.begin() + a, h.perm.begin() + b);
    for (int i = 0; i < b - a; ++i) {
      h.geom[a + i] = tg[idx[i]];
      h.perm[a + i] = tp[idx[i]];
    }
  }
  // per-visibility tap phase exp(i (om_y + om_x) / 2) of the frequencies
  // taken in [-pi, pi), in sorted order (FP64 on the host)
  h.vph.resize(n);
  for (int64_t p = 0; p < n; ++p) {
    const int64_t m = h.perm[p];
    const double oyn = om_y[m] - 2.0 * M_PI * std::floor((om_y[m] + M_PI) / (2.0 * M_PI));
    const double oxn = om_x[m] - 2.0 * M_PI * std::floor((om_x[m] + M_PI) / (2.0 * M_PI));
    const double ph = 0.5 * (oyn + oxn);
    h.vph[p] = make_float2((float)std::cos(ph), (float)std::sin(ph));
  }
  // Gridding order: inside each sub-bin, the visibilities grouped by 2x2
  // block of start cells (block-major, stable), as positions in the sorted
  // order above; the gridding kernel accumulates one block's 8x8 patch in
  // registers.
  h.gperm.resize(n);
  for (int k = 0; k < op->nkeys; ++k) {
    const int a = h.sb_off[k], b = h.sb_off[k + 1];
    int cnt[17] = {0};
    auto block_of = [&](int i) {
      unsigned kp;
      std::memcpy(&kp, &h.geom[i].z, sizeof(kp));
      return (int)(((kp & 7u) >> 1) | ((((kp >> 14) & 7u) >> 1) << 2));
    };
    for (int i = a; i < b; ++i) cnt[block_of(i) + 1]++;
    for (int t = 0; t < 16; ++t) cnt[t + 1] += cnt[t];
    for (int i = a; i < b; ++i) h.gperm[a + cnt[block_of(i)]++] = i;
  }
  h.set = true;
}

// Work lists for the tile kernels.  Degridding: one item per non-empty
// (channel, tile), split into slices of at most kDegridSlice visibilities.
// Gridding: one item per (channel, tile) whose footprint ring holds any
// visibility, split into slices of at most op->grid_slice; split tiles get partial
// tiles that grid_combine_kernel sums.  Empty tiles are never written (the
// gridding output is zeroed at commit).  Items run channel by channel in tile
// order, so neighbouring tiles (which share aprons) run close together.
constexpr int kDegridSlice = 8192;

static void build_work_lists(MeasOp* op, cudaStream_t s) {
  const int L = op->L, nt = op->ntiles();
  const int S = kSubPerTile;
  auto key = [&](int sb0, int sb1) {
    return ((sb1 / S) * op->nT0 + sb0 / S) * (S * S) + (sb1 % S) * S + (sb0 % S);
  };
  std::vector<WorkItem> dg, gr;
  std::vector<int> gr_work;   // visibilities an item grids (own + ring)
  std::vector<GridPlan> plans;
  std::vector<GridCombine> comb;
  op->h_dg_off.assign(L + 1, 0);
  op->h_gr_off.assign(L + 1, 0);
  op->h_comb_off.assign(L + 1, 0);
  int pslot = 0;
  for (int c = 0; c < L; ++c) {
    const std::vector<int32_t>& off = op->ch[c].sb_off;
    for (int t = 0; t < nt; ++t) {
      const int t0 = t % op->nT0, t1 = t / op->nT0;
      const int own = off[(t + 1) * S * S] - off[t * S * S];
      if (own > 0) {
        const int ns = (own + kDegridSlice - 1) / kDegridSlice;
        for (int k = 0; k < ns; ++k) {
          dg.push_back(WorkItem{c, t, k, ns, (int)dg.size(), 0});
        }
      }
      // visibilities starting in the tile or in the 8-cell ring left/above it
      int ring = 0;
      const int sbc1 = (t1 * S - 1 + op->nsb1) % op->nsb1, sbr0 = (t0 * S - 1 + op->nsb0) % op->nsb0;
      const int r_end = std::min(t0 * S + S, op->nsb0), c_end = std::min(t1 * S + S, op->nsb1);
      for (int sb0 = t0 * S; sb0 < r_end; ++sb0) ring += off[key(sb0, sbc1) + 1] - off[key(sb0, sbc1)];
      for (int sb1 = t1 * S; sb1 < c_end; ++sb1) ring += off[key(sbr0, sb1) + 1] - off[key(sbr0, sb1)];
      ring += off[key(sbr0, sbc1) + 1] - off[key(sbr0, sbc1)];
      const int tot = own + ring;
      if (tot == 0) continue;
      // sub-bin schedule: phases by parity, largest first (ties by index)
      GridPlan plan{};
      {
        const int nrows = std::min(S, op->nsb0 - t0 * S), ncols = std::min(S, op->nsb1 - t1 * S);
        std::vector<std::pair<int, int>> ph[4];   // (-size, sub-bin index)
        for (int j = -1; j < S; ++j)
          for (int i = -1; i < S; ++i) {
            if (i >= nrows || j >= ncols) continue;
            const int sb0 = i < 0 ? sbr0 : t0 * S + i, sb1 = j < 0 ? sbc1 : t1 * S + j;
            const int len = off[key(sb0, sb1) + 1] - off[key(sb0, sb1)];
            if (len == 0) continue;
            ph[((i + 1) & 1) | (((j + 1) & 1) << 1)].push_back({-len, (j + 1) * (S + 1) + (i + 1)});
          }
        int pos = 0;
        for (int q = 0; q < 4; ++q) {
          std::sort(ph[q].begin(), ph[q].end());
          plan.count[q] = (int)ph[q].size();
          for (const auto& e : ph[q]) plan.sub[pos++] = (uint8_t)e.second;
        }
      }
      const int ns = (tot + op->grid_slice - 1) / op->grid_slice;
      if (ns == 1) {
        gr.push_back(WorkItem{c, t, 0, 1, -1, 0});
        gr_work.push_back(tot);
        plans.push_back(plan);
      } else {
        comb.push_back(GridCombine{c, t, pslot, ns});
        for (int k = 0; k < ns; ++k) {
          gr.push_back(WorkItem{c, t, k, ns, pslot + k, 0});
          gr_work.push_back(tot / ns);
          plans.push_back(plan);
        }
        pslot += ns;
      }
    }
    op->h_dg_off[c + 1] = (int)dg.size();
    op->h_gr_off[c + 1] = (int)gr.size();
    op->h_comb_off[c + 1] = (int)comb.size();
  }
  op->dg_items.alloc(std::max<size_t>(dg.size(), 1));
  op->dg_items.upload(dg.data(), dg.size(), s);
  op->gr_items.alloc(std::max<size_t>(gr.size(), 1));
  op->gr_items.upload(gr.data(), gr.size(), s);
  // launch order of the whole-operator gridding: largest item first (ties:
  // item order), so the long dense tiles start at once and the short ones
  // fill in behind them
  std::vector<int> gord(gr.size());
  for (size_t k = 0; k < gord.size(); ++k) gord[k] = (int)k;
  std::stable_sort(gord.begin(), gord.end(), [&](int u, int v) { return gr_work[u] > gr_work[v]; });
  op->gr_order.alloc(std::max<size_t>(gord.size(), 1));
  op->gr_order.upload(gord.data(), gord.size(), s);
  op->gr_plan.alloc(std::max<size_t>(plans.size(), 1));
  op->gr_plan.upload(plans.data(), plans.size(), s);
  op->gr_combine.alloc(std::max<size_t>(comb.size(), 1));
  op->gr_combine.upload(comb.data(), comb.size(), s);
  op->dg_off.alloc(L + 1);
  op->dg_off.upload(op->h_dg_off.data(), L + 1, s);
  op->gr_partial.alloc(std::max<size_t>((size_t)pslot * kTileCells * kTileCells, 1));
  op->partials.alloc(std::max<size_t>(dg.size(), 1) * kMaxBlocksPerChannel * 2);
  FHS_CUDA(cudaStreamSynchronize(s));
}

void measop_set_grid_slice(MeasOp* op, int slice) {
  FHS_CHECK(slice >= 1024, FHS_ERR_INVALID_ARG, "gridding slice below 1024 visibilities");
  if (op->dr || slice == op->grid_slice) return;
  DeviceGuard g(op->device);
  FHS_CUDA(cudaStreamSynchronize(op->stream));
  op->grid_slice = slice;
  build_work_lists(op, op->stream);
  ++op->layout_epoch;
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
  // a DR operator (measop_create_dr) has no visibility geometry: its data
  // entries are grid cells, in order (perm = identity)
  if (!op->dr) {
    op->geom.alloc(std::max<int64_t>(op->Mtot, 1));
    op->sb_off.alloc((size_t)L * (op->nkeys + 1));
  }
  op->zbuf.alloc(std::max<int64_t>(op->Mtot, 1));
  op->perm.alloc(std::max<int64_t>(op->Mtot, 1));
  if (!op->dr) {
    op->gperm.alloc(std::max<int64_t>(op->Mtot, 1));
    op->vph.alloc(std::max<int64_t>(op->Mtot, 1));
  }
  for (int c = 0; c < L; ++c) {
    const ChannelHost& h = op->ch[c];
    if (h.M) {
      if (!op->dr) {
        FHS_CUDA(cudaMemcpyAsync(op->geom.p + op->h_voff[c], h.geom.data(), h.M * sizeof(float4),
                                 cudaMemcpyHostToDevice, s));
        FHS_CUDA(cudaMemcpyAsync(op->gperm.p + op->h_voff[c], h.gperm.data(), h.M * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, s));
        FHS_CUDA(cudaMemcpyAsync(op->vph.p + op->h_voff[c], h.vph.data(), h.M * sizeof(float2),
                                 cudaMemcpyHostToDevice, s));
      }
      FHS_CUDA(cudaMemcpyAsync(op->perm.p + op->h_voff[c], h.perm.data(), h.M * sizeof(int32_t),
                               cudaMemcpyHostToDevice, s));
    }
    if (!op->dr)
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
  if (op->dr)
    measop_dr_lists(op, s);
  else
    build_work_lists(op, s);
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
  if (measop_own_fft(op)) measop_fft_tables(op, s);   // the hand-written transforms of fft.cu
  FHS_CUDA(cudaStreamSynchronize(s));
  // host copies of the sorted geometry are no longer needed
  for (auto& h : op->ch) {
    std::vector<float4>().swap(h.geom);
    std::vector<int32_t>().swap(h.perm);
    std::vector<int32_t>().swap(h.gperm);
    std::vector<float2>().swap(h.vph);
  }
  op->committed = true;
}

__global__ void pad_real_kernel(const float* __restrict__ x, float* __restrict__ pad, const float* __restrict__ sy,
                                const float* __restrict__ sx, int Ny, int Nx, int Ky, int Kx, int p0) {
  const int64_t N = (int64_t)Ny * Nx;
  const int plane = blockIdx.y;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(p / Ny), iy = (int)(p - (int64_t)ix * Ny);
    int ky = iy - Ny / 2;
    ky += ky < 0 ? Ky : 0;
    int kx = ix - Nx / 2;
    kx += kx < 0 ? Kx : 0;
    pad[(size_t)(p0 + plane) * Ky * Kx + (size_t)kx * Ky + ky] = x[(size_t)plane * N + p] * sy[iy] * sx[ix];
  }
}

void measop_enable_r2c(MeasOp* op) {
  if (op->plan_r2c || op->own_fft) return;
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  if (op->tw_y.p) {   // the hand-written transforms of fft.cu (tables built at commit)
    op->imgr.alloc((size_t)op->L * op->Npix());
    op->own_fft = true;
    FHS_CUDA(cudaStreamSynchronize(s));
    return;
  }
  op->padr.alloc((size_t)op->L * op->No());
  op->padr.zero(s);
  op->imgr.alloc((size_t)op->L * op->No());
  int n[2] = {op->Kx, op->Ky};
  FHS_CUFFT(cufftPlanMany(&op->plan_r2c, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, op->L));
  FHS_CUFFT(cufftSetStream(op->plan_r2c, s));
  FHS_CUFFT(cufftPlanMany(&op->plan_c2r, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, op->L));
  FHS_CUFFT(cufftSetStream(op->plan_c2r, s));
  FHS_CUDA(cudaStreamSynchronize(s));
}

// H(k) = (B(k) + conj(B(-k))) / 2 on the half plane k0 <= Ky/2: the
// Hermitian part of the gridded spectrum, whose complex-to-real inverse FFT
// is Re(IFFT(B)), the only part the adjoint keeps.
__global__ void hermitian_half_kernel(const float2* __restrict__ B, float2* __restrict__ H, int Ky, int Kx) {
  const int Kh = Ky / 2 + 1;
  const int plane = blockIdx.z;
  const int k1 = blockIdx.y;
  const int m1 = k1 == 0 ? 0 : Kx - k1;
  const float2* b = B + (size_t)plane * Kx * Ky;
  float2* h = H + (size_t)plane * Kx * Kh;
  for (int k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < Kh; k0 += gridDim.x * blockDim.x) {
    const float2 u = b[(size_t)k1 * Ky + k0];
    const float2 v = b[(size_t)m1 * Ky + (k0 == 0 ? 0 : Ky - k0)];
    h[(size_t)k1 * Kh + k0] = make_float2(0.5f * (u.x + v.x), 0.5f * (u.y - v.y));
  }
}

void fft_inverse_c2r(const MeasOp* op, cudaStream_t s) {
  FHS_CHECK(op->plan_c2r, FHS_ERR_STATE, "real-to-complex path not enabled");
  const int Kh = op->Ky / 2 + 1;
  dim3 grid(ceil_div(Kh, 256), op->Kx, op->L);
  hermitian_half_kernel<<<grid, 256, 0, s>>>(op->gridB.p, op->gridA.p, op->Ky, op->Kx);
  count_launch();
  FHS_LAUNCH_CHECK();
  FHS_CUFFT(cufftExecC2R(op->plan_c2r, (cufftComplex*)op->gridA.p, op->imgr.p));
}

void solver_fft_forward(const MeasOp* op, const float* x, cudaStream_t s) {
  if (op->own_fft) {
    const int step = op->fft_chunk > 0 ? op->fft_chunk : op->L;
    for (int p0 = 0; p0 < op->L; p0 += step)
      fft_forward_half(op, x + (size_t)p0 * op->Npix(), p0, std::min(step, op->L - p0), s);
  } else {
    fft_forward_r2c(op, s);   // reads the padded image written by the caller
  }
}

void solver_fft_inverse(const MeasOp* op, cudaStream_t s) {
  if (op->own_fft) {
    const int step = op->fft_chunk > 0 ? op->fft_chunk : op->L;
    for (int p0 = 0; p0 < op->L; p0 += step)
      fft_inverse_real(op, op->imgr.p + (size_t)p0 * op->Npix(), p0, std::min(step, op->L - p0), s);
  } else {
    fft_inverse_c2r(op, s);
  }
}

__global__ void scale_image_kernel(float* __restrict__ img, const float* __restrict__ sy,
                                   const float* __restrict__ sx, int Ny, int Nx) {
  const int64_t N = (int64_t)Ny * Nx;
  float* p = img + (size_t)blockIdx.y * N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i / Ny), iy = (int)(i - (int64_t)ix * Ny);
    p[i] *= sy[iy] * sx[ix];
  }
}

void launch_scale_image(const MeasOp* op, float* img, int np, cudaStream_t s) {
  dim3 grid(grid_blocks(op->Npix(), 256), np);
  scale_image_kernel<<<grid, 256, 0, s>>>(img, op->sy.p, op->sx.p, op->Ny, op->Nx);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_pad_real(const MeasOp* op, const float* x, int p0, int np, cudaStream_t s) {
  FHS_CHECK(op->plan_r2c, FHS_ERR_STATE, "real-to-complex path not enabled");
  dim3 grid(grid_blocks(op->Npix(), 256), np);
  pad_real_kernel<<<grid, 256, 0, s>>>(x, op->padr.p, op->sy.p, op->sx.p, op->Ny, op->Nx, op->Ky, op->Kx, p0);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void fft_forward_r2c(const MeasOp* op, cudaStream_t s) {
  (void)s;
  FHS_CHECK(op->plan_r2c, FHS_ERR_STATE, "real-to-complex path not enabled");
  FHS_CUFFT(cufftExecR2C(op->plan_r2c, op->padr.p, (cufftComplex*)op->gridA.p));
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

PrecondView MeasOp::precond_view(const double2* w) const {
  PrecondView v;
  v.pu = pu.p;
  v.w = w;
  v.mu = blk_mu.p;
  return v;
}

void launch_degrid_plain(const MeasOp* op, int c0, int nc, float2* out, cudaStream_t s, bool half) {
  if (op->dr) return launch_dr_apply(op, 0, c0, nc, nullptr, out, nullptr, nullptr, nullptr, s, half);
  const int i0 = op->h_dg_off[c0], n = op->h_dg_off[c0 + nc] - i0;
  if (n == 0) return;
  if (half)
    degrid_kernel<7, 0, 1, true><<<n, 256, 0, s>>>(op->view(), op->gridA.p, op->dg_items.p, nullptr, i0, out,
                                                   nullptr, nullptr, nullptr, nullptr, nullptr, PrecondView{});
  else
    degrid_kernel<7, 0, 1, false><<<n, 256, 0, s>>>(op->view(), op->gridA.p, op->dg_items.p, nullptr, i0, out,
                                                    nullptr, nullptr, nullptr, nullptr, nullptr, PrecondView{});
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_grid_plain(const MeasOp* op, int c0, int nc, const float2* v, cudaStream_t s) {
  if (op->dr) return launch_dr_apply(op, 3, c0, nc, v, nullptr, nullptr, nullptr, nullptr, s, false);
  launch_grid_kernel<7, 0>(op, c0, nc, v, nullptr, nullptr, nullptr, PrecondView{}, s);
}

void launch_crop_real(const MeasOp* op, float* out, const float* sigma, int p0, int np, cudaStream_t s) {
  dim3 grid(grid_blocks(op->Npix(), 256), np);
  crop_real_kernel<<<grid, 256, 0, s>>>(op->gridA.p, out, sigma, op->sy.p, op->sx.p, op->Ny, op->Nx, op->Ky,
                                        op->Kx, p0);
  count_launch();
  FHS_LAUNCH_CHECK();
}

template <int MODE, int NB>
static void degrid_dual(const MeasOp* op, int i0, int n, const float2* v2, float2* gold, const float2* y,
                        PrecondView pc, cudaStream_t s, bool half) {
  if (half)
    degrid_kernel<7, MODE, NB, true><<<n, 256, 0, s>>>(op->view(), op->gridA.p, op->dg_items.p, nullptr, i0,
                                                       nullptr, v2, gold, y, op->partials.p, op->zbuf.p, pc);
  else
    degrid_kernel<7, MODE, NB, false><<<n, 256, 0, s>>>(op->view(), op->gridA.p, op->dg_items.p, nullptr, i0,
                                                        nullptr, v2, gold, y, op->partials.p, op->zbuf.p, pc);
  count_launch();
  FHS_LAUNCH_CHECK();
}

// the fewest per-thread block accumulators that cover every channel
template <int MODE>
static void degrid_dual_nb(const MeasOp* op, int c0, int nc, const float2* v2, float2* gold, const float2* y,
                           PrecondView pc, cudaStream_t s, bool half) {
  const int i0 = op->h_dg_off[c0], n = op->h_dg_off[c0 + nc] - i0;
  if (n == 0) return;
  int nb = 1;
  for (int c = c0; c < c0 + nc; ++c) nb = std::max(nb, (int)op->h_nblk[c]);
  if (nb <= 1)
    degrid_dual<MODE, 1>(op, i0, n, v2, gold, y, pc, s, half);
  else if (nb <= 2)
    degrid_dual<MODE, 2>(op, i0, n, v2, gold, y, pc, s, half);
  else if (nb <= 4)
    degrid_dual<MODE, 4>(op, i0, n, v2, gold, y, pc, s, half);
  else if (nb <= 6)
    degrid_dual<MODE, 6>(op, i0, n, v2, gold, y, pc, s, half);
  else if (nb <= 8)
    degrid_dual<MODE, 8>(op, i0, n, v2, gold, y, pc, s, half);
  else
    degrid_dual<MODE, 16>(op, i0, n, v2, gold, y, pc, s, half);
}

void launch_degrid_dual(const MeasOp* op, int c0, int nc, float2* v2, float2* gold, const float2* y,
                        cudaStream_t s, bool half) {
  if (op->dr) return launch_dr_apply(op, 1, c0, nc, nullptr, nullptr, v2, gold, y, s, half);
  degrid_dual_nb<1>(op, c0, nc, v2, gold, y, PrecondView{}, s, half);
}

void launch_degrid_dual_precond(const MeasOp* op, int c0, int nc, const float2* v2, float2* gold,
                                const float2* y, const double2* w, cudaStream_t s, bool half) {
  FHS_CHECK(op->precond, FHS_ERR_STATE, "no preconditioner set");
  degrid_dual_nb<2>(op, c0, nc, v2, gold, y, op->precond_view(w), s, half);
}

static void block_reduce(const MeasOp* op, int c0, int nc, int mode, cudaStream_t s) {
  dim3 grid(nc, kMaxBlocksPerChannel);
  block_reduce_kernel<<<grid, 256, 0, s>>>(op->partials.p, op->dg_off.p, c0, op->ch_nblk.p, op->ch_blkoff.p,
                                           op->blk_eps.p, op->blk_scale.p, op->blk_stats.p, mode,
                                           op->fb_c.p, op->fb_iter.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_block_reduce(const MeasOp* op, int c0, int nc, cudaStream_t s) { block_reduce(op, c0, nc, 0, s); }

void launch_block_reduce_precond(const MeasOp* op, int c0, int nc, cudaStream_t s) {
  block_reduce(op, c0, nc, 1, s);
}

void launch_grid_dual(const MeasOp* op, int c0, int nc, float2* v2, cudaStream_t s) {
  if (op->dr) return launch_dr_apply(op, 2, c0, nc, nullptr, nullptr, v2, nullptr, nullptr, s, false);
  launch_grid_kernel<7, 1>(op, c0, nc, nullptr, v2, op->blk_scale.p, op->zbuf.p, PrecondView{}, s);
}

void launch_grid_dual_precond(const MeasOp* op, int c0, int nc, float2* v2, const double2* w, cudaStream_t s) {
  FHS_CHECK(op->precond, FHS_ERR_STATE, "no preconditioner set");
  launch_grid_kernel<7, 2>(op, c0, nc, nullptr, v2, nullptr, op->zbuf.p, op->precond_view(w), s);
}

}  // namespace fhs
