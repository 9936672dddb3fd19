// Visibility gridding (dimensionality reduction, DR) on B200 (sm_100a).
//
// Replaces the DR measurement operator of
// lib/operators/util_load_data_gen_dr_measurement_operator.m:109-228 and its
// application in src/update_dual_data_fidelity.m:85-125,
// lib/operators/HS_forward_operator_G.m:41-45, HS_adjoint_operator_G.m:46-49
// and src/compute_residual_images.m:42-80:
//   H = G^H G (the reference keeps tril(H) with its diagonal halved and
//   applies H u + (u' H)'), W = diag(H) > 0, Lambda = diag(H)^-1/2 on W,
//   forward  y = Lambda .* (H Fx)(W),  adjoint  g2(W) = H (Lambda .* y).
// The grids here carry the centring phase rho_k (the image sits at
// (n - N/2) mod K, see measop.cu): Fx = rho Fx_ref and G = G_ref conj(rho),
// so this H is rho H_ref conj(rho).  The per-cell weight kept on the device
// is omega_k = Lambda_k conj(rho_k): forward y = omega (H Fx), adjoint stages
// u = conj(omega) y, and the data space matches the reference's exactly.
//
// Two cells couple only when one visibility's 7 x 7 support holds both, so H
// is a 13 x 13 stencil on the (periodic) oversampled grid.  It is stored as
// its half T on the active cells only, per channel [85][n_c] c64 (plane j,
// data index i): T[i][0] = H_kk / 2 and T[i][d] = H(k, k + d) for the 84
// offsets with d1 < 0 or (d1 == 0, d0 < 0), so that H u = T u + T^H u:
//   (H u)[k] = 2 Re(T[k][0]) u[k] + sum_d T[k][d] u[k + d] + conj(T[k - d][d]) u[k - d]
// (rows of inactive cells are zero and not stored).  The apply kernel is a
// gather (no atomics): a CTA stages u and the cell -> data index map over a
// 64 x 16 cell tile and its 6-cell apron in shared memory; per offset each
// thread loads T of its 4 cells and of their neighbours k - d (index from the
// staged map) together, 8 independent loads in flight, since the kernel
// waits on global-load latency.  Tiles without active cells skip the loop.
// The data space of channel c is its active cells in column-major order, the
// order of MATLAB's Fx(W); solver vectors (y, v2, G Fx_old, z) live there.
//
// H is built on the device in FP64 from the committed visibility operator,
// one channel at a time into a dense [85][Ky Kx] scratch: one CTA per 8 x 8
// cell block gathers the visibilities of the 2 x 2 sub-bins whose supports
// can reach the block, each thread owning a fixed set of (cell, offset) sums
// (deterministic, no atomics); the active rows are then gathered into the
// compact store.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "cplx.cuh"
#include "measop.cuh"

namespace fhs {

namespace {

constexpr int kDrTileY = 64;  // cells along Ky (contiguous) per apply tile
constexpr int kDrTileX = 16;  // cells along Kx
constexpr int kDrSY = kDrTileY + 2 * kDrReach;  // 76 staged rows
constexpr int kDrSX = kDrTileX + 2 * kDrReach;  // 28 staged columns

// offset j of the half stencil: j = 0 the diagonal, 1..78 d1 in [-6, -1] x
// d0 in [-6, 6], 79..84 d1 = 0, d0 in [-6, -1]
__host__ __device__ __forceinline__ void dr_offset(int j, int& d0, int& d1) {
  if (j == 0) {
    d0 = d1 = 0;
    return;
  }
  const int q = j - 1;
  const int side = 2 * kDrReach + 1;
  if (q < kDrReach * side) {
    d1 = q / side - kDrReach;
    d0 = q % side - kDrReach;
  } else {
    d1 = 0;
    d0 = q - kDrReach * side - kDrReach;
  }
}

// ------------------------------------------------------------------ build
constexpr int kBuildThreads = 512;
constexpr int kBuildGroups = kBuildThreads / (kBinCells * kBinCells);    // 8 offset groups per cell
constexpr int kBuildSlots = (kDrHalf + kBuildGroups - 1) / kBuildGroups;  // 11 offsets per thread
constexpr int kBuildChunk = 64;                                           // visibilities staged at once

__global__ void __launch_bounds__(kBuildThreads) dr_build_kernel(OpView op, int c0, float2* __restrict__ T,
                                                                 double* __restrict__ diag) {
  __shared__ float2 s_hy[kBuildChunk][8], s_hx[kBuildChunk][8];
  __shared__ float s_w2[kBuildChunk];
  __shared__ int s_s0[kBuildChunk], s_s1[kBuildChunk];
  const int ch = c0 + blockIdx.z;
  const int B0 = blockIdx.x * kBinCells, B1 = blockIdx.y * kBinCells;
  const int cell = threadIdx.x % (kBinCells * kBinCells);
  const int grp = threadIdx.x / (kBinCells * kBinCells);
  const int k0 = B0 + cell % kBinCells, k1 = B1 + cell / kBinCells;
  double2 acc[kBuildSlots];
#pragma unroll
  for (int i = 0; i < kBuildSlots; ++i) acc[i] = make_double2(0.0, 0.0);
  const int32_t* off = op.sb_off + (size_t)ch * (op.nkeys + 1);
  const int64_t vo = op.ch_voff[ch];
  constexpr int S = kSubPerTile;
  for (int src = 0; src < 4; ++src) {
    const int sb0 = (blockIdx.x + op.nsb0 - 1 + (src & 1)) % op.nsb0;
    const int sb1 = (blockIdx.y + op.nsb1 - 1 + (src >> 1)) % op.nsb1;
    const int key = ((sb1 / S) * op.nT0 + sb0 / S) * (S * S) + (sb1 % S) * S + (sb0 % S);
    const int beg = off[key], end = off[key + 1];
    for (int c = beg; c < end; c += kBuildChunk) {
      const int n = min(kBuildChunk, end - c);
      __syncthreads();
      if (threadIdx.x < n) {
        const float4 gm = op.geom[vo + c + threadIdx.x];
        float2 hy[7], hx[7];
        taps<7>(op.py, fabsf(gm.x), hy);   // the sign bit of the stored offsets is a wrap flag
        taps<7>(op.px, fabsf(gm.y), hx);
#pragma unroll
        for (int a = 0; a < 7; ++a) {
          s_hy[threadIdx.x][a] = hy[a];
          s_hx[threadIdx.x][a] = hx[a];
        }
        const unsigned kp = __float_as_uint(gm.z);
        s_s0[threadIdx.x] = (int)(kp & 0x3FFFu);
        s_s1[threadIdx.x] = (int)((kp >> 14) & 0x3FFFu);
        s_w2[threadIdx.x] = gm.w * gm.w;
      }
      __syncthreads();
      for (int v = 0; v < n; ++v) {
        const int a = wrap(k0 - s_s0[v], op.Ky), b = wrap(k1 - s_s1[v], op.Kx);
        if (a > 6 || b > 6) continue;
        // conj(G[m, k]) = w conj(hy[a] hx[b]); G[m, k + d] = w hy[a + d0] hx[b + d1]
        const float2 ga = s_hy[v][a], gb = s_hx[v][b];
        const double gr = (double)ga.x * gb.x - (double)ga.y * gb.y;
        const double gi = (double)ga.x * gb.y + (double)ga.y * gb.x;
        const double w2 = s_w2[v];
#pragma unroll
        for (int i = 0; i < kBuildSlots; ++i) {
          const int j = grp + kBuildGroups * i;
          if (j >= kDrHalf) break;
          int d0, d1;
          dr_offset(j, d0, d1);
          const int a2 = a + d0, b2 = b + d1;
          if (a2 < 0 || a2 > 6 || b2 < 0 || b2 > 6) continue;
          const float2 ha = s_hy[v][a2], hb = s_hx[v][b2];
          const double pr = (double)ha.x * hb.x - (double)ha.y * hb.y;
          const double pi = (double)ha.x * hb.y + (double)ha.y * hb.x;
          acc[i].x += w2 * (gr * pr + gi * pi);
          acc[i].y += w2 * (gr * pi - gi * pr);
        }
      }
    }
  }
  const int64_t No = (int64_t)op.Ky * op.Kx;
  const int64_t k = (int64_t)k1 * op.Ky + k0;
#pragma unroll
  for (int i = 0; i < kBuildSlots; ++i) {
    const int j = grp + kBuildGroups * i;
    if (j >= kDrHalf) break;
    float2 t = make_float2((float)acc[i].x, (float)acc[i].y);
    if (j == 0) {
      diag[(size_t)blockIdx.z * No + k] = acc[i].x;
      t = make_float2((float)(0.5 * acc[i].x), 0.f);  // H_kk is real
    }
    T[((size_t)blockIdx.z * kDrHalf + j) * No + k] = t;
  }
}

// compact store of one channel: Tc[j][i] = dense[j][cell_i]
__global__ void dr_compact_kernel(const float2* __restrict__ dense, const int32_t* __restrict__ cells, int64_t n,
                                  int64_t No, float2* __restrict__ Tc) {
  const int j = blockIdx.y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    Tc[j * n + i] = dense[j * No + cells[i]];
}

// ------------------------------------------------------------------ apply
// MODE 0: out(W) = omega (H u), u = Fx.  MODE 1: l2-ball dual pass 1 (u = Fx;
// hf = omega (H u), z = v2 + 2 hf - gold - y -> zbuf, hf -> gold, FP64 sums
// ||z||^2, ||hf - y||^2).  MODE 2: dual pass 2 (u = conj(omega) scale z;
// gridB = H u; v2 = scale z on W).  MODE 3: gridB = H u, u = conj(omega) vin.
// HALF: u is read from the R2C half spectrum [Kx][Ky/2 + 1].
struct DrView {
  const float2* const* T;  // [L] per-channel stencil [85][n_c]
  const float2* omega;
  const int32_t* map;
  const int64_t* ch_voff;
  const float* blk_scale;
  const int32_t* ch_M;
  int Ky, Kx, tiles_y, tiles;
};

struct DrSmem {
  float2 su[kDrSX][kDrSY];              // operand u over the tile and its 6-cell apron
  int32_t sm[kDrSX][kDrSY];             // data index of each staged cell, -1 off W
  double red[2][8];
};

template <int MODE, bool HALF>
__global__ void __launch_bounds__(256) dr_apply_kernel(DrView dv, int c0, const float2* __restrict__ gridA,
                                                       const float2* __restrict__ vin, float2* __restrict__ out,
                                                       float2* __restrict__ gridB, float2* __restrict__ v2,
                                                       float2* __restrict__ gold, const float2* __restrict__ y,
                                                       float2* __restrict__ zbuf, double* __restrict__ partials) {
  extern __shared__ __align__(16) unsigned char dr_smem_raw[];
  DrSmem& S = *reinterpret_cast<DrSmem*>(dr_smem_raw);
  const int ch = c0 + blockIdx.y;
  const int tile = blockIdx.x;
  const int B0 = (tile % dv.tiles_y) * kDrTileY, B1 = (tile / dv.tiles_y) * kDrTileX;
  const int Ky = dv.Ky, Kx = dv.Kx;
  const int64_t No = (int64_t)Ky * Kx;
  const float2* omega = dv.omega + (size_t)ch * No;
  const int32_t* map = dv.map + (size_t)ch * No;
  const int64_t vo = dv.ch_voff[ch];
  const float scale = MODE == 2 ? dv.blk_scale[(size_t)ch * kMaxBlocksPerChannel] : 1.f;
  const int ty = threadIdx.x % kDrTileY, tx = threadIdx.x / kDrTileY;  // 4 column groups
  const int k0 = B0 + ty;
  // stage u and the index map over the tile and its apron (periodic grid)
  const int Kh = Ky / 2 + 1;
  const float2* g = gridA + (size_t)ch * (HALF ? Kh : Ky) * Kx;
  int own = 0;
  for (int idx = threadIdx.x; idx < kDrSX * kDrSY; idx += blockDim.x) {
    const int cx = idx / kDrSY, cy = idx - cx * kDrSY;
    const int q0 = wrap(B0 - kDrReach + cy, Ky), q1 = wrap(B1 - kDrReach + cx, Kx);
    const int64_t q = (int64_t)q1 * Ky + q0;
    const int i = map[q];
    S.sm[cx][cy] = i;
    if (i >= 0 && cx >= kDrReach && cx < kDrReach + kDrTileX && cy >= kDrReach && cy < kDrReach + kDrTileY)
      own = 1;
    float2 u;
    if (MODE <= 1) {
      if (!HALF) {
        u = __ldg(g + (size_t)q1 * Ky + q0);
      } else if (q0 < Kh) {
        u = __ldg(g + (size_t)q1 * Kh + q0);
      } else {  // Hermitian mirror
        const float2 m = __ldg(g + (size_t)(q1 == 0 ? 0 : Kx - q1) * Kh + (Ky - q0));
        u = make_float2(m.x, -m.y);
      }
    } else {
      u = make_float2(0.f, 0.f);
      if (i >= 0) {
        const float2 z = MODE == 2 ? zbuf[vo + i] : vin[vo + i];
        u = cmulc(omega[q], make_float2(scale * z.x, scale * z.y));
      }
    }
    S.su[cx][cy] = u;
  }
  own = __syncthreads_or(own);
  float2 acc[kDrTileX / 4];
#pragma unroll
  for (int r = 0; r < kDrTileX / 4; ++r) acc[r] = make_float2(0.f, 0.f);
  if (own) {
    // per offset, the 4 cells of a thread issue their 8 stencil loads together
    // (the kernel waits on global loads: memory-level parallelism per thread)
    const int64_t n = dv.ch_M[ch];
    const float2* Tc = dv.T[ch];
    int ia[kDrTileX / 4];
#pragma unroll
    for (int r = 0; r < kDrTileX / 4; ++r) {
      const int lx = tx + 4 * r;
      ia[r] = S.sm[lx + kDrReach][ty + kDrReach];
      if (ia[r] >= 0) {
        const float2 t0 = __ldg(Tc + ia[r]);
        const float2 uk = S.su[lx + kDrReach][ty + kDrReach];
        acc[r] = make_float2(2.f * t0.x * uk.x, 2.f * t0.x * uk.y);
      }
    }
#pragma unroll 2
    for (int j = 1; j < kDrHalf; ++j) {
      int d0, d1;
      dr_offset(j, d0, d1);
      const float2* Tj = Tc + j * n;
      float2 a[kDrTileX / 4], b[kDrTileX / 4];
#pragma unroll
      for (int r = 0; r < kDrTileX / 4; ++r) {
        const int lx = tx + 4 * r;
        const int ib = S.sm[lx + kDrReach - d1][ty + kDrReach - d0];  // neighbour k - d
        a[r] = ia[r] >= 0 ? __ldg(Tj + ia[r]) : make_float2(0.f, 0.f);
        b[r] = ib >= 0 && ia[r] >= 0 ? __ldg(Tj + ib) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int r = 0; r < kDrTileX / 4; ++r) {
        const int lx = tx + 4 * r;
        acc[r] = cfma(a[r], S.su[lx + kDrReach + d1][ty + kDrReach + d0], acc[r]);
        acc[r] = cfma(make_float2(b[r].x, -b[r].y), S.su[lx + kDrReach - d1][ty + kDrReach - d0], acc[r]);
      }
    }
  }
  double nz = 0.0, nr = 0.0;
#pragma unroll
  for (int r = 0; r < kDrTileX / 4; ++r) {
    const int lx = tx + 4 * r;
    const int k1 = B1 + lx;
    if (k0 >= Ky || k1 >= Kx) continue;
    const int64_t k = (int64_t)k1 * Ky + k0;
    const int i = S.sm[lx + kDrReach][ty + kDrReach];
    if (MODE == 0) {
      if (i >= 0) out[vo + i] = cmul(omega[k], acc[r]);
    } else if (MODE == 1) {
      if (i >= 0) {
        const float2 hf = cmul(omega[k], acc[r]);
        const float2 yv = y[vo + i], vv = v2[vo + i], go = gold[vo + i];
        const float2 z = make_float2(vv.x + 2.f * hf.x - go.x - yv.x, vv.y + 2.f * hf.y - go.y - yv.y);
        zbuf[vo + i] = z;
        gold[vo + i] = hf;
        const float2 rr = make_float2(hf.x - yv.x, hf.y - yv.y);
        nz += (double)z.x * z.x + (double)z.y * z.y;
        nr += (double)rr.x * rr.x + (double)rr.y * rr.y;
      }
    } else {
      gridB[(size_t)ch * No + k] = acc[r];  // exactly 0 off W
      if (MODE == 2 && i >= 0) {
        const float2 z = zbuf[vo + i];
        v2[vo + i] = make_float2(scale * z.x, scale * z.y);
      }
    }
  }
  if (MODE == 1) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      nz += __shfl_down_sync(0xffffffffu, nz, o);
      nr += __shfl_down_sync(0xffffffffu, nr, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      S.red[0][w] = nz;
      S.red[1][w] = nr;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      double t = 0.0;
      for (int q = 0; q < 8; ++q) t += S.red[threadIdx.x][q];
      partials[((size_t)ch * dv.tiles + tile) * kMaxBlocksPerChannel * 2 + threadIdx.x] = t;
    }
  }
}

template <int MODE, bool HALF>
void dr_launch(dim3 grid, cudaStream_t s, const DrView& dv, int c0, const float2* gA, const float2* vin,
               float2* out, float2* gB, float2* v2, float2* gold, const float2* y, float2* zb, double* pa) {
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(dr_apply_kernel<MODE, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(DrSmem)));
    attr[dev] = true;
  }
  dr_apply_kernel<MODE, HALF><<<grid, 256, sizeof(DrSmem), s>>>(dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
}

}  // namespace

void launch_dr_apply(const MeasOp* op, int mode, int c0, int nc, const float2* vin, float2* out, float2* v2,
                     float2* gold, const float2* y, cudaStream_t s, bool half) {
  FHS_CHECK(op->dr, FHS_ERR_STATE, "not a dimensionality-reduced operator");
  if (nc <= 0) return;
  DrView dv;
  dv.T = op->dr_Tptr.p;
  dv.ch_M = op->ch_M.p;
  dv.omega = op->dr_omega.p;
  dv.map = op->dr_map.p;
  dv.ch_voff = op->ch_voff.p;
  dv.blk_scale = op->blk_scale.p;
  dv.Ky = op->Ky;
  dv.Kx = op->Kx;
  dv.tiles_y = (op->Ky + kDrTileY - 1) / kDrTileY;
  dv.tiles = op->dr_tiles;
  dim3 grid(op->dr_tiles, nc);
  const float2* gA = op->gridA.p;
  float2* gB = op->gridB.p;
  float2* zb = op->zbuf.p;
  double* pa = op->partials.p;
  switch (mode) {
    case 0:
      if (half)
        dr_launch<0, true>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      else
        dr_launch<0, false>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      break;
    case 1:
      if (half)
        dr_launch<1, true>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      else
        dr_launch<1, false>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      break;
    case 2:
      dr_launch<2, false>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      break;
    default:
      dr_launch<3, false>(grid, s, dv, c0, gA, vin, out, gB, v2, gold, y, zb, pa);
      break;
  }
  count_launch();
  FHS_LAUNCH_CHECK();
}

// Partial-sum slots of the DR dual: one per (channel, apply tile), read by the
// block reduction through the per-channel slot offsets.
void measop_dr_lists(MeasOp* op, cudaStream_t s) {
  const int L = op->L;
  op->h_dg_off.assign(L + 1, 0);
  op->h_gr_off.assign(L + 1, 0);
  op->h_comb_off.assign(L + 1, 0);
  for (int c = 0; c <= L; ++c) op->h_dg_off[c] = c * op->dr_tiles;
  op->dg_items.alloc(1);
  op->gr_items.alloc(1);
  op->gr_combine.alloc(1);
  op->gr_partial.alloc(1);
  op->dg_off.alloc(L + 1);
  op->dg_off.upload(op->h_dg_off.data(), L + 1, s);
  op->partials.alloc((size_t)std::max(L * op->dr_tiles, 1) * kMaxBlocksPerChannel * 2);
  op->partials.zero(s);
}

MeasOp* measop_create_dr(const MeasOp* vis) {
  FHS_CHECK(vis != nullptr && vis->committed, FHS_ERR_STATE, "commit the visibility operator first");
  FHS_CHECK(!vis->dr, FHS_ERR_INVALID_ARG, "operator is already dimensionality-reduced");
  FHS_CHECK(vis->Jy == 7 && vis->Jx == 7, FHS_ERR_UNSUPPORTED, "DR supports 7x7 interpolation kernels");
  // offsets up to +-6 must stay distinct on the periodic grid
  FHS_CHECK(vis->Ky >= 16 && vis->Kx >= 16, FHS_ERR_UNSUPPORTED, "DR needs oversampled grids of at least 16x16");
  const int L = vis->L;
  const int64_t No = vis->No();
  MeasOp* op = measop_create(vis->device, vis->Ny, vis->Nx, vis->Ky / vis->Ny, vis->Kx / vis->Nx, 7, 7, L);
  try {
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    FHS_CUDA(cudaStreamSynchronize(vis->stream));
    op->dr = true;
    op->dr_tiles = ((op->Ky + kDrTileY - 1) / kDrTileY) * ((op->Kx + kDrTileX - 1) / kDrTileX);
    op->dr_omega.alloc((size_t)L * No);
    op->dr_map.alloc((size_t)L * No);
    op->dr_Tc.resize(L);
    DevBuf<float2> dense;   // one channel's stencil over the whole grid
    dense.alloc((size_t)kDrHalf * No);
    DevBuf<double> diag;
    diag.alloc((size_t)No);
    DevBuf<int32_t> dcell;
    std::vector<double> hd((size_t)No);
    std::vector<float2> hl((size_t)No);
    std::vector<int32_t> hm((size_t)No);
    std::vector<int32_t> cells;
    std::vector<float2*> tptr(L, nullptr);
    const OpView v = vis->view();
    for (int c = 0; c < L; ++c) {
      dim3 grid(vis->nsb0, vis->nsb1, 1);
      dr_build_kernel<<<grid, kBuildThreads, 0, s>>>(v, c, dense.p, diag.p);
      count_launch();
      FHS_LAUNCH_CHECK();
      diag.download(hd.data(), No, s);
      FHS_CUDA(cudaStreamSynchronize(s));
      // W = diag(H) > 0, Lambda = diag(H)^-1/2
      // (util_load_data_gen_dr_measurement_operator.m:213-216); omega = Lambda conj(rho)
      ChannelHost& h = op->ch[c];
      h.perm.clear();
      const size_t first = cells.size();
      int32_t n = 0;
      for (int64_t k = 0; k < No; ++k) {
        if (hd[k] > 0) {
          hm[k] = n++;
          const double lam = 1.0 / std::sqrt(hd[k]);
          const int64_t k1 = k / op->Ky, k0 = k - k1 * op->Ky;
          // rho_k = exp(i pi (k0 Ny / Ky + k1 Nx / Kx)), arguments reduced mod 2
          const double a = (double)((k0 * op->Ny) % (2 * (int64_t)op->Ky)) / op->Ky +
                           (double)((k1 * op->Nx) % (2 * (int64_t)op->Kx)) / op->Kx;
          hl[k] = make_float2((float)(lam * std::cos(M_PI * a)), (float)(-lam * std::sin(M_PI * a)));
          cells.push_back((int32_t)k);
        } else {
          hm[k] = -1;
          hl[k] = make_float2(0.f, 0.f);
        }
      }
      h.M = n;
      h.block_sizes.assign(1, n);
      h.perm.resize(n);
      std::iota(h.perm.begin(), h.perm.end(), 0);
      h.set = true;
      FHS_CUDA(cudaMemcpyAsync(op->dr_omega.p + (size_t)c * No, hl.data(), No * sizeof(float2),
                               cudaMemcpyHostToDevice, s));
      FHS_CUDA(cudaMemcpyAsync(op->dr_map.p + (size_t)c * No, hm.data(), No * sizeof(int32_t),
                               cudaMemcpyHostToDevice, s));
      if (n > 0) {
        op->dr_Tc[c].reset(new DevBuf<float2>());
        op->dr_Tc[c]->alloc((size_t)kDrHalf * n);
        tptr[c] = op->dr_Tc[c]->p;
        if (dcell.n < (size_t)n) dcell.alloc(n);
        dcell.upload(cells.data() + first, n, s);
        dim3 cg((unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), kDrHalf);
        dr_compact_kernel<<<cg, 256, 0, s>>>(dense.p, dcell.p, n, No, tptr[c]);
        count_launch();
        FHS_LAUNCH_CHECK();
      }
      FHS_CUDA(cudaStreamSynchronize(s));
    }
    op->dr_Tptr.alloc(L);
    op->dr_Tptr.upload(tptr.data(), L, s);
    op->dr_cell.alloc(std::max<size_t>(cells.size(), 1));
    op->dr_cell.upload(cells.data(), cells.size(), s);
    measop_commit(op);
  } catch (...) {
    delete op;
    throw;
  }
  return op;
}

}  // namespace fhs
