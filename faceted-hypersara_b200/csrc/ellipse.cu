// Preconditioned data-fidelity dual on B200: the ellipsoid projection of
// solver_proj_elipse_fb (RI-measurement-operator submodule, called at
// src/update_dual_data_fidelity.m:133-135 and src/sara/sara.m:561,594) and the
// uniform-weight preconditioner of util_gen_preconditioning_matrix
// (imaging/imaging.m:436-438, default_parameters.json "preconditioning").
//
// Per block b of channel l the dual step projects s = v2/pU + r2 onto the
// ball ||z - y|| <= eps in the metric diag(1/pU):
//   proj = argmin_z (z - s)^H diag(1/pU) (z - s)  s.t. ||z - y|| <= eps,
// by forward-backward splitting (Onose et al. 2017):
//   z_k = P_B(z_{k-1} - mu (z_{k-1} - s) / pU),   mu = min over the block of pU,
// stopping when ||z_k - z_{k-1}|| <= stop ||z_k|| (k >= min_itr) or at max_itr,
// then v2 = v2 + pU (r2 - proj) = pU (s - proj).
// In the centred variables w = z - y and d = s - y one step reads
//   t_k - y = w_{k-1} + (mu/pU)(d - w_{k-1}),   w_k = c_k (t_k - y),
//   c_k = min(1, eps / ||t_k - y||),
// so an iteration is one streaming pass over the block's visibilities and one
// block reduction.  The pass that writes w_k also reduces ||t_{k+1} - y||^2
// (next scale), ||w_k - w_{k-1}||^2 and ||w_k + y||^2 (stopping test): one
// pass plus one small finalise kernel per iteration.  The first scale comes
// from the degridding pass (degrid_kernel MODE 2), the final v2 from the
// gridding pass (grid_kernel MODE 2).  w is kept in FP64 because the default
// stopping tolerance (1e-8) lies below FP32 resolution.  Blocks that stopped
// skip their visibilities; the launch sequence itself is fixed (max_itr
// passes) so one iteration stays capturable in a CUDA graph.
#include "measop.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace fhs {

namespace {

constexpr int kFbThreads = 256;
constexpr int kFbWarps = kFbThreads / 32;
constexpr int kFbChunk = 8192;  // visibilities per CTA and pass
constexpr int kFbUnroll = 4;    // visibilities in flight per thread

int blocks_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

// t - y = w + m (d - w), m = mu / pU (the gradient step in centred form)
__device__ __forceinline__ double2 fb_point(double2 w, float2 d, double m) {
  return make_double2(fma(m, (double)d.x - w.x, w.x), fma(m, (double)d.y - w.y, w.y));
}

template <int NB>
__global__ void __launch_bounds__(kFbThreads) fb_advance_kernel(
    const FbItem* __restrict__ items, int item0, const int64_t* __restrict__ ch_voff,
    const uint8_t* __restrict__ vblk, const float* __restrict__ pu, const float2* __restrict__ dbuf,
    const float2* __restrict__ y, double2* __restrict__ w, const float* __restrict__ blk_mu,
    const double* __restrict__ fb_c, const int* __restrict__ fb_iter, double* __restrict__ part) {
  __shared__ float s_mu[kMaxBlocksPerChannel];
  __shared__ double s_c[kMaxBlocksPerChannel];
  __shared__ int s_act[kMaxBlocksPerChannel];
  __shared__ int any;
  __shared__ double red[kFbWarps][NB * 3];
  const FbItem it = items[item0 + blockIdx.x];
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  if (threadIdx.x < kMaxBlocksPerChannel) {
    const size_t k = (size_t)it.ch * kMaxBlocksPerChannel + threadIdx.x;
    const int a = fb_iter[k] >= 0 ? 1 : 0;
    s_act[threadIdx.x] = a;
    s_mu[threadIdx.x] = blk_mu[k];
    s_c[threadIdx.x] = fb_c[k];
    if (a) atomicOr(&any, 1);
  }
  __syncthreads();
  if (!any) return;  // every block of the channel has stopped (uniform across the CTA)
  // ||t - y||^2 sets the next scale: FP64 (its rounding must not jitter the
  // iterate); the stopping-test sums only need FP32 per thread
  double acc0[NB];
  float acc1[NB], acc2[NB];
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    acc0[k] = 0.0;
    acc1[k] = acc2[k] = 0.f;
  }
  const int64_t vo = ch_voff[it.ch];
  // kFbUnroll visibilities per thread and step: their loads are issued
  // together (the block id first, then the operands of the active ones)
  for (int base = it.beg + threadIdx.x; base < it.end; base += kFbThreads * kFbUnroll) {
    int bl[kFbUnroll];
    bool act[kFbUnroll];
#pragma unroll
    for (int u = 0; u < kFbUnroll; ++u) {
      const int i = base + u * kFbThreads;
      bl[u] = i < it.end ? (int)vblk[vo + i] : 0;
    }
#pragma unroll
    for (int u = 0; u < kFbUnroll; ++u) act[u] = (base + u * kFbThreads < it.end) && s_act[bl[u]];
    float ip[kFbUnroll];
    float2 d[kFbUnroll], yv[kFbUnroll];
    double2 wp[kFbUnroll];
#pragma unroll
    for (int u = 0; u < kFbUnroll; ++u) {
      if (act[u]) {
        const int64_t i = vo + base + u * kFbThreads;
        ip[u] = pu[i];
        d[u] = dbuf[i];
        wp[u] = w[i];
        yv[u] = y[i];
      }
    }
#pragma unroll
    for (int u = 0; u < kFbUnroll; ++u) {
      if (!act[u]) continue;
      const int b = bl[u];
      const float inv = 1.f / ip[u];
      const double m = (double)s_mu[b] * (double)inv;
      const double c = s_c[b];
      const double2 t = fb_point(wp[u], d[u], m);
      const double2 wn = make_double2(c * t.x, c * t.y);
      w[vo + base + u * kFbThreads] = wn;
      const double2 tn = fb_point(wn, d[u], m);
      const double dx = wn.x - wp[u].x, dy = wn.y - wp[u].y;
      const double zx = wn.x + (double)yv[u].x, zy = wn.y + (double)yv[u].y;
      const double q0 = tn.x * tn.x + tn.y * tn.y;
      const float q1 = (float)(dx * dx + dy * dy), q2 = (float)(zx * zx + zy * zy);
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        if (b == k) {
          acc0[k] += q0;
          acc1[k] += q1;
          acc2[k] += q2;
        }
      }
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NB; ++k) {
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      double v = f == 0 ? acc0[k] : (double)(f == 1 ? acc1[k] : acc2[k]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][k * 3 + f] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < NB * 3) {
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < kFbWarps; ++q) v += red[q][threadIdx.x];
    part[(size_t)(item0 + blockIdx.x) * kMaxBlocksPerChannel * 3 + threadIdx.x] = v;
  }
}

// One CTA per (channel, block): sums the pass's partials in a fixed order,
// applies the stopping test and sets the scale of the next projection.
__global__ void __launch_bounds__(256) fb_finalize_kernel(const double* __restrict__ part,
                                                          const int* __restrict__ fb_off, int c0,
                                                          const int32_t* __restrict__ ch_nblk,
                                                          const double* __restrict__ blk_eps,
                                                          double* __restrict__ fb_c, int* __restrict__ fb_iter,
                                                          int* __restrict__ fb_count, int min_itr, int max_itr,
                                                          double stop) {
  const int ch = c0 + blockIdx.x, b = blockIdx.y;
  if (b >= ch_nblk[ch]) return;
  const size_t k = (size_t)ch * kMaxBlocksPerChannel + b;
  const int done = fb_iter[k];
  if (done < 0) return;
  __shared__ double s0[256], s1[256], s2[256];
  double a0 = 0, a1 = 0, a2 = 0;
  for (int t = fb_off[ch] + threadIdx.x; t < fb_off[ch + 1]; t += blockDim.x) {
    const double* p = part + ((size_t)t * kMaxBlocksPerChannel + b) * 3;
    a0 += p[0];
    a1 += p[1];
    a2 += p[2];
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  s2[threadIdx.x] = a2;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      s0[threadIdx.x] += s0[threadIdx.x + h];
      s1[threadIdx.x] += s1[threadIdx.x + h];
      s2[threadIdx.x] += s2[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int itn = done + 1;
    const double tn = sqrt(s0[0]), dn = sqrt(s1[0]), zn = sqrt(s2[0]);
    if ((itn >= min_itr && dn <= stop * zn) || itn >= max_itr) {
      fb_iter[k] = -1;
      fb_count[k] = itn;
    } else {
      fb_iter[k] = itn;
      const double eps = blk_eps[k];
      fb_c[k] = tn > eps ? eps / tn : 1.0;
    }
  }
}

__global__ void vblk_kernel(const float4* __restrict__ geom, uint8_t* __restrict__ vblk, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    vblk[i] = (uint8_t)(__float_as_uint(geom[i].z) >> 28);
}

__global__ void pu_gather_kernel(const float* __restrict__ in, float* __restrict__ out,
                                 const int32_t* __restrict__ perm, int64_t vo, int M) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x)
    out[vo + i] = in[perm[vo + i]];
}

// w = z - y (z in the original order, interleaved complex double; NULL = 0)
__global__ void w_from_proj_kernel(const double* __restrict__ z, const float2* __restrict__ y,
                                   double2* __restrict__ w, const int32_t* __restrict__ perm,
                                   const int64_t* __restrict__ ch_voff, const int32_t* __restrict__ ch_M) {
  const int ch = blockIdx.y;
  const int64_t vo = ch_voff[ch];
  const int M = ch_M[ch];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 yv = y[vo + i];
    double zx = 0.0, zy = 0.0;
    if (z) {
      const int64_t src = vo + perm[vo + i];
      zx = z[2 * src];
      zy = z[2 * src + 1];
    }
    w[vo + i] = make_double2(zx - (double)yv.x, zy - (double)yv.y);
  }
}

__global__ void proj_from_w_kernel(const double2* __restrict__ w, const float2* __restrict__ y,
                                   double* __restrict__ z, const int32_t* __restrict__ perm,
                                   const int64_t* __restrict__ ch_voff, const int32_t* __restrict__ ch_M) {
  const int ch = blockIdx.y;
  const int64_t vo = ch_voff[ch];
  const int M = ch_M[ch];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t dst = vo + perm[vo + i];
    const double2 wv = w[vo + i];
    const float2 yv = y[vo + i];
    z[2 * dst] = wv.x + (double)yv.x;
    z[2 * dst + 1] = wv.y + (double)yv.y;
  }
}

__global__ void scale_pu_kernel(float2* __restrict__ v, const float* __restrict__ pu, int64_t n, int root) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float s = root ? sqrtf(pu[i]) : pu[i];
    float2 a = v[i];
    a.x *= s;
    a.y *= s;
    v[i] = a;
  }
}

void fb_setup(MeasOp* op, cudaStream_t s) {
  const int L = op->L;
  op->pu.alloc(std::max<int64_t>(op->Mtot, 1));
  op->vblk.alloc(std::max<int64_t>(op->Mtot, 1));
  if (op->Mtot > 0) {
    vblk_kernel<<<blocks_for(op->Mtot), 256, 0, s>>>(op->geom.p, op->vblk.p, op->Mtot);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
  op->h_mu.assign((size_t)L * kMaxBlocksPerChannel, 1.f);
  op->blk_mu.alloc((size_t)L * kMaxBlocksPerChannel);
  op->fb_c.alloc((size_t)L * kMaxBlocksPerChannel);
  op->fb_c.zero(s);
  op->fb_iter.alloc((size_t)L * kMaxBlocksPerChannel);
  FHS_CUDA(cudaMemsetAsync(op->fb_iter.p, 0xFF, op->fb_iter.n * sizeof(int), s));  // -1: no pass pending
  op->fb_count.alloc((size_t)L * kMaxBlocksPerChannel);
  op->fb_count.zero(s);
  std::vector<FbItem> items;
  op->h_fb_off.assign(L + 1, 0);
  op->max_nblk = 1;
  for (int c = 0; c < L; ++c) {
    const int M = op->h_M[c];
    for (int b = 0; b < M; b += kFbChunk) items.push_back(FbItem{c, b, std::min(M, b + kFbChunk), 0});
    op->h_fb_off[c + 1] = (int)items.size();
    op->max_nblk = std::max(op->max_nblk, (int)op->h_nblk[c]);
  }
  op->fb_items.alloc(std::max<size_t>(items.size(), 1));
  op->fb_items.upload(items.data(), items.size(), s);
  op->fb_off.alloc(L + 1);
  op->fb_off.upload(op->h_fb_off.data(), L + 1, s);
  op->fb_part.alloc(std::max<size_t>(items.size(), 1) * kMaxBlocksPerChannel * 3);
  op->pu_set.assign(L, 0);
}

template <int NB>
void advance(const MeasOp* op, int i0, int n, double2* w, const float2* y, cudaStream_t s) {
  fb_advance_kernel<NB><<<n, kFbThreads, 0, s>>>(op->fb_items.p, i0, op->ch_voff.p, op->vblk.p, op->pu.p,
                                                 op->zbuf.p, y, w, op->blk_mu.p, op->fb_c.p, op->fb_iter.p,
                                                 op->fb_part.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace

void measop_set_preconditioner(MeasOp* op, int c, const double* pu) {
  FHS_CHECK(op->committed, FHS_ERR_STATE, "commit the operator before setting a preconditioner");
  // util_load_data_gen_dr_measurement_operator.m:118: no preconditioning with DR
  FHS_CHECK(!op->dr, FHS_ERR_UNSUPPORTED, "no preconditioner on a dimensionality-reduced operator");
  FHS_CHECK(c >= 0 && c < op->L, FHS_ERR_INVALID_ARG, "bad channel index");
  const int M = op->h_M[c];
  FHS_CHECK(M == 0 || pu != nullptr, FHS_ERR_INVALID_ARG, "null preconditioner");
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  if (op->pu_set.empty()) fb_setup(op, s);
  std::vector<float> h(M);
  const std::vector<int64_t>& bs = op->ch[c].block_sizes;
  int64_t pos = 0;
  for (size_t b = 0; b < bs.size(); ++b) {
    float mn = std::numeric_limits<float>::infinity();
    for (int64_t m = pos; m < pos + bs[b]; ++m) {
      FHS_CHECK(std::isfinite(pu[m]) && pu[m] > 0, FHS_ERR_INVALID_ARG, "preconditioner entries must be finite and > 0");
      h[m] = (float)pu[m];
      FHS_CHECK(h[m] > 0.f, FHS_ERR_INVALID_ARG, "preconditioner entry below FP32 range");
      mn = std::min(mn, h[m]);
    }
    op->h_mu[(size_t)c * kMaxBlocksPerChannel + b] = bs[b] > 0 ? mn : 1.f;
    pos += bs[b];
  }
  if (M > 0) {
    DevBuf<float> tmp;
    tmp.alloc(M);
    tmp.upload(h.data(), M, s);
    pu_gather_kernel<<<blocks_for(M), 256, 0, s>>>(tmp.p, op->pu.p, op->perm.p, op->h_voff[c], M);
    count_launch();
    FHS_LAUNCH_CHECK();
    FHS_CUDA(cudaStreamSynchronize(s));
  }
  op->blk_mu.upload(op->h_mu.data(), op->h_mu.size(), s);
  FHS_CUDA(cudaStreamSynchronize(s));
  op->pu_set[c] = 1;
  op->precond = std::all_of(op->pu_set.begin(), op->pu_set.end(), [](char v) { return v != 0; });
}

void launch_fb_iterations(const MeasOp* op, int c0, int nc, double2* w, const float2* y, int max_itr,
                          int min_itr, double stop, cudaStream_t s) {
  FHS_CHECK(op->precond, FHS_ERR_STATE, "no preconditioner set");
  FHS_CHECK(max_itr >= 1, FHS_ERR_INVALID_ARG, "elipse_proj_max_iter must be >= 1");
  const int i0 = op->h_fb_off[c0], n = op->h_fb_off[c0 + nc] - i0;
  const int nb = op->max_nblk;
  for (int k = 0; k < max_itr; ++k) {
    if (n > 0) {
      // per-thread accumulators for every block of a channel: the fewest that fit
      if (nb <= 1)
        advance<1>(op, i0, n, w, y, s);
      else if (nb <= 2)
        advance<2>(op, i0, n, w, y, s);
      else if (nb <= 3)
        advance<3>(op, i0, n, w, y, s);
      else if (nb <= 4)
        advance<4>(op, i0, n, w, y, s);
      else if (nb <= 6)
        advance<6>(op, i0, n, w, y, s);
      else if (nb <= 8)
        advance<8>(op, i0, n, w, y, s);
      else
        advance<16>(op, i0, n, w, y, s);
    }
    fb_finalize_kernel<<<dim3(nc, kMaxBlocksPerChannel), 256, 0, s>>>(
        op->fb_part.p, op->fb_off.p, c0, op->ch_nblk.p, op->blk_eps.p, op->fb_c.p, op->fb_iter.p,
        op->fb_count.p, min_itr, max_itr, stop);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
}

void launch_w_from_proj(const MeasOp* op, const double* z, const float2* y, double2* w, cudaStream_t s) {
  if (op->maxM <= 0) return;
  dim3 grid(blocks_for(op->maxM), op->L);
  w_from_proj_kernel<<<grid, 256, 0, s>>>(z, y, w, op->perm.p, op->ch_voff.p, op->ch_M.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_proj_from_w(const MeasOp* op, const double2* w, const float2* y, double* z, cudaStream_t s) {
  if (op->maxM <= 0) return;
  dim3 grid(blocks_for(op->maxM), op->L);
  proj_from_w_kernel<<<grid, 256, 0, s>>>(w, y, z, op->perm.p, op->ch_voff.p, op->ch_M.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void launch_scale_pu(const MeasOp* op, float2* v, bool root, cudaStream_t s) {
  FHS_CHECK(op->precond, FHS_ERR_STATE, "no preconditioner set");
  if (op->Mtot <= 0) return;
  scale_pu_kernel<<<blocks_for(op->Mtot), 256, 0, s>>>(v, op->pu.p, op->Mtot, root ? 1 : 0);
  count_launch();
  FHS_LAUNCH_CHECK();
}

// util_gen_preconditioning_matrix (uniform weighting): pU = 1 / (number of
// visibilities in the same cell of a (Ky sub) x (Kx sub) grid), cells centred
// on the grid points.  Host code: it runs once per data set.
void gen_uniform_weights(int64_t n, const double* om_y, const double* om_x, int Ky, int Kx, int sub, double* pu) {
  FHS_CHECK(n >= 0 && Ky > 0 && Kx > 0 && sub >= 1, FHS_ERR_INVALID_ARG, "bad sizes");
  const int64_t gy = (int64_t)Ky * sub, gx = (int64_t)Kx * sub;
  FHS_CHECK(gy * gx <= ((int64_t)1 << 31), FHS_ERR_UNSUPPORTED, "counting grid larger than 2^31 cells");
  FHS_CHECK(n == 0 || (om_y && om_x && pu), FHS_ERR_INVALID_ARG, "null argument");
  std::vector<int64_t> cell(n);
  std::vector<int32_t> cnt((size_t)(gy * gx), 0);
  for (int64_t m = 0; m < n; ++m) {
    FHS_CHECK(std::isfinite(om_y[m]) && std::isfinite(om_x[m]), FHS_ERR_NUMERIC, "non-finite frequency");
    int64_t ky = (int64_t)std::floor(om_y[m] * (double)gy / (2.0 * M_PI) + 0.5) % gy;
    int64_t kx = (int64_t)std::floor(om_x[m] * (double)gx / (2.0 * M_PI) + 0.5) % gx;
    if (ky < 0) ky += gy;
    if (kx < 0) kx += gx;
    cell[m] = ky + gy * kx;
    cnt[(size_t)cell[m]]++;
  }
  for (int64_t m = 0; m < n; ++m) pu[m] = 1.0 / (double)cnt[(size_t)cell[m]];
}

}  // namespace fhs
