// Primal-dual iteration of facetHyperSARA / hyperSARA / sara on B200.
//
// One iteration (src/fhs/facetHyperSARA.m:701-783, src/hs/hyperSARA.m:565-617,
// src/sara/sara.m:521-637) is a fixed launch sequence on one stream, captured
// once into a CUDA graph and replayed:
//   primal update + scaled zero-padded image for the FFT   (fhs_update_primal.m:33-38)
//   FFT, degridding + l2-ball dual (pass 1), block norms,
//   dual scaling + gridding (pass 2), inverse FFT          (update_dual_data_fidelity.m:116-147)
//   SARA analysis of xhat, l21 prox, synthesis            (fhs_update_dual_sparsity.m:67-93)
//   facet Gram, FP64 eigensolve, rank-L update            (fhs_update_dual_lowrankness.m:40-45)
//   g = sigma00 sum_q D_q v0_q + sigma11 Psi v1 + sigma22 Re(At G^H v2)
//   FP64 statistics into a device ring (rel_x, ||x||, residual, eps, priors).
// The host reads the ring once per iteration only when it evaluates the
// stopping rule (facetHyperSARA.m:877-881) and reweights (:952-1137).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>

#include "apikern.cuh"
#include "solver.cuh"

namespace fhs {

namespace {

constexpr int kPrimalBlocks = 128;

__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x / 32, ln = threadIdx.x % 32;
  if (ln == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x / 32;
    a = ln < nw ? sa[ln] : 0.0;
    b = ln < nw ? sb[ln] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
}

__global__ void __launch_bounds__(256) primal_pad_kernel(float* __restrict__ x, const float* __restrict__ g,
                                                         float* __restrict__ xhat, float* __restrict__ pad,
                                                         const float* __restrict__ sy, const float* __restrict__ sx,
                                                         int Ny, int Nx, int Ky, int Kx, double* __restrict__ part) {
  const int plane = blockIdx.y;
  const int64_t N = (int64_t)Ny * Nx;
  float* xp = x + (size_t)plane * N;
  const float* gp = g + (size_t)plane * N;
  float* hp = xhat + (size_t)plane * N;
  float* pp = pad ? pad + (size_t)plane * Ky * Kx : nullptr;
  double a = 0.0, b = 0.0;
  // four pixels per step (N is a multiple of 4: Ny and Nx are even), float4
  // loads and stores of x, g and xhat for memory-level parallelism
  const int64_t N4 = N / 4;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N4; q += (int64_t)gridDim.x * blockDim.x) {
    const float4 xo4 = reinterpret_cast<const float4*>(xp)[q];
    const float4 g4 = reinterpret_cast<const float4*>(gp)[q];
    const float xo[4] = {xo4.x, xo4.y, xo4.z, xo4.w};
    const float gv[4] = {g4.x, g4.y, g4.z, g4.w};
    float xn[4], xh[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      xn[e] = fmaxf(xo[e] - gv[e], 0.f);
      xh[e] = 2.f * xn[e] - xo[e];
      const double d = (double)xo[e] - xn[e];
      a += d * d;
      b += (double)xn[e] * xn[e];
      if (pad) {   // the padded image of the cuFFT path (the hand-written FFT reads x)
        const int64_t p = 4 * q + e;
        const int ix = (int)(p / Ny), iy = (int)(p - (int64_t)ix * Ny);
        int ky = iy - Ny / 2;
        ky += ky < 0 ? Ky : 0;
        int kx = ix - Nx / 2;
        kx += kx < 0 ? Kx : 0;
        pp[(size_t)kx * Ky + ky] = xn[e] * sy[iy] * sx[ix];
      }
    }
    reinterpret_cast<float4*>(xp)[q] = make_float4(xn[0], xn[1], xn[2], xn[3]);
    reinterpret_cast<float4*>(hp)[q] = make_float4(xh[0], xh[1], xh[2], xh[3]);
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    part[((size_t)plane * gridDim.x + blockIdx.x) * 2] = a;
    part[((size_t)plane * gridDim.x + blockIdx.x) * 2 + 1] = b;
  }
}

struct AssembleArgs {
  int Ny, Nx, Ky, Kx, lg, Qy, nuclear;
  int img_compact;   // img holds [L][Nx][Ny] (hand-written FFT) instead of [L][Kx][Ky]
  float sigma00;
  const NucFacet* facets;
  const float* wy;
  const float* wx;
  const int* cover_y;
  const int* cover_x;
  int64_t v0_group;
};

// g = sigma22 s Re(At(...)) + sigma11 Psi v1 (in g1) + sigma00 sum_q D_q v0_q.
// One thread per pixel walks every channel plane: the pixel's facets (up to
// four overlapping ones), their window values and dual offsets are looked up
// once and reused by all L planes; each plane's accesses stay coalesced
// across the warp (consecutive pixels of a column).
__global__ void __launch_bounds__(256) assemble_kernel(AssembleArgs a, int L, float* __restrict__ g,
                                                       const float* __restrict__ img, const float* __restrict__ g1,
                                                       const float* __restrict__ v0, const float* __restrict__ sigma22,
                                                       const float* __restrict__ sy, const float* __restrict__ sx) {
  const int64_t N = (int64_t)a.Ny * a.Nx;
  const int64_t plane_img = (int64_t)a.Ky * a.Kx;  // Re(IFFT(gridB)) planes, [Kx][Ky]
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(p / a.Ny), iy = (int)(p - (int64_t)ix * a.Ny);
    int ky = iy - a.Ny / 2;
    ky += ky < 0 ? a.Ky : 0;
    int kx = ix - a.Nx / 2;
    kx += kx < 0 ? a.Kx : 0;
    const int64_t kimg = a.img_compact ? p : (int64_t)kx * a.Ky + ky;
    const int64_t pstride = a.img_compact ? N : plane_img;
    const float syi = sy[iy], sxi = sx[ix];
    int ne = 0;
    int64_t base[4], P[4];
    float w[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      base[e] = 0;
      P[e] = 0;
      w[e] = 0.f;
    }
    if (a.nuclear) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int qy = a.cover_y[2 * iy + i];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int qx = a.cover_x[2 * ix + j];
          if (qy < 0 || qx < 0) continue;
          const NucFacet f = a.facets[qx * a.Qy + qy];
          const int ny = f.y1 - f.y0;
          const int ly = iy - f.y0, lx = ix - f.x0;
          const int slot = 2 * i + j;
          base[slot] = f.v0_off + (int64_t)lx * ny + ly;
          P[slot] = (int64_t)ny * (f.x1 - f.x0);
          w[slot] = a.wy[f.wy_off + ly] * a.wx[f.wx_off + lx];
          ne |= 1 << slot;
        }
      }
    }
    for (int plane = 0; plane < L; ++plane) {
      const int grp = plane / a.lg, lc = plane - grp * a.lg;
      float val = sigma22[plane] * syi * sxi * img[(size_t)plane * pstride + kimg] + g1[(size_t)plane * N + p];
      if (ne) {
        float acc = 0.f;
        const float* vg = v0 + (int64_t)grp * a.v0_group;
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (ne & (1 << e)) acc = fmaf(w[e], vg[base[e] + (int64_t)lc * P[e]], acc);
        val = fmaf(a.sigma00, acc, val);
      }
      g[(size_t)plane * N + p] = val;
    }
  }
}

// One CTA per spectral group reduces the iteration's FP64 statistics into the
// device ring; the last CTA to finish advances the ring counter.
__global__ void __launch_bounds__(256) stats_kernel(const double* __restrict__ primal_part, int nparts, int lg, int G,
                                                    const double* __restrict__ blk_stats,
                                                    const int32_t* __restrict__ ch_nblk,
                                                    const int32_t* __restrict__ ch_blkoff,
                                                    const double* __restrict__ blk_eps,
                                                    const double* __restrict__ nuc_vals, int Q,
                                                    const double* __restrict__ l21_part, int prox_blocks,
                                                    const double* __restrict__ l21_acc, double* __restrict__ ring,
                                                    int* __restrict__ counter, int* __restrict__ done) {
  __shared__ double red[6][256];
  __shared__ int last;
  const int g = blockIdx.x;
  const int c = *counter;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int k = threadIdx.x; k < lg * nparts; k += blockDim.x) {
    const int l = g * lg + k / nparts, kk = k % nparts;
    v[0] += primal_part[((size_t)l * nparts + kk) * 2];
    v[1] += primal_part[((size_t)l * nparts + kk) * 2 + 1];
  }
  for (int l = g * lg + threadIdx.x; l < (g + 1) * lg; l += blockDim.x)
    for (int b = 0; b < ch_nblk[l]; ++b) {
      v[2] += blk_stats[2 * (ch_blkoff[l] + b) + 1];
      const double e = blk_eps[(size_t)l * kMaxBlocksPerChannel + b];
      v[3] += e * e;
    }
  if (nuc_vals)
    for (int q = threadIdx.x; q < Q; q += blockDim.x) v[4] += nuc_vals[g * Q + q];
  for (int k = threadIdx.x; k < prox_blocks; k += blockDim.x) v[5] += l21_part[(size_t)g * prox_blocks + k];
  if (threadIdx.x == 0) v[5] += l21_acc[g];
  for (int f = 0; f < 6; ++f) red[f][threadIdx.x] = v[f];
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int f = 0; f < 6; ++f) red[f][threadIdx.x] += red[f][threadIdx.x + s];
    __syncthreads();
  }
  double* rec = ring + (size_t)(c % kReportRing) * G * kReportFields;
  if (threadIdx.x < 6) rec[g * kReportFields + threadIdx.x] = red[threadIdx.x][0];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(done, 1) == G - 1);
  __syncthreads();
  if (last && threadIdx.x == 0) {
    *done = 0;
    *counter = c + 1;
  }
}

__global__ void weights_kernel(const float* __restrict__ norms, int64_t s, const double* __restrict__ ups,
                               float* __restrict__ w) {
  const int g = blockIdx.y;
  const double u = ups[g];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (int64_t)gridDim.x * blockDim.x) {
    const double d = norms[(size_t)g * s + i];
    w[(size_t)g * s + i] = (u + d) > 0 ? (float)(u / (u + d)) : 1.f;
  }
}

__global__ void weights0_kernel(const double* __restrict__ sigma, int n, const double* __restrict__ ups,
                                double* __restrict__ w0) {
  const int id = blockIdx.x;  // g*Q + q
  const double u = ups[id];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = sigma[(size_t)id * n + i];
    w0[(size_t)id * n + i] = (u + d) > 0 ? u / (u + d) : 1.0;
  }
}

__global__ void diff_norm_kernel(const float* __restrict__ a, const float* __restrict__ b, int64_t n,
                                 double* __restrict__ out) {
  double d2 = 0, a2 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double d = (double)a[i] - b[i];
    d2 += d * d;
    a2 += (double)a[i] * a[i];
  }
  block_sum2(d2, a2);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = d2;
    out[2 * blockIdx.x + 1] = a2;
  }
}

int nblk(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

}  // namespace

Solver::~Solver() {
  if (graph) cudaGraphExecDestroy(graph);
}

static const char* kStageNames[] = {"primal_pad", "fft_forward", "degrid_dual", "block_reduce", "ellipse_fb",
                                    "grid_dual",
                                    "fft_inverse", "sara_analysis_prox", "l21_prox", "sara_synthesis", "facet_gram",
                                    "facet_eig", "facet_reconstruct", "assemble_g", "stats"};
constexpr int kStages = sizeof(kStageNames) / sizeof(kStageNames[0]);

// Records ev[k] after stage k-1 (ev[0] before the first) when ev is non-null.
static void solver_launch_iteration(Solver* S, cudaStream_t s, cudaEvent_t* ev = nullptr) {
  MeasOp* op = S->op;
  const int L = S->L;
  int stage = 0;
  auto mark = [&]() {
    if (ev) FHS_CUDA(cudaEventRecord(ev[stage], s));
    ++stage;
  };
  mark();
  primal_pad_kernel<<<dim3(kPrimalBlocks, L), 256, 0, s>>>(S->x.p, S->g.p, S->xhat.p,
                                                           op->own_fft ? nullptr : op->padr.p, op->sy.p,
                                                           op->sx.p, S->Ny, S->Nx, op->Ky, op->Kx, S->primal_part.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  mark();
  solver_fft_forward(op, S->x.p, s);
  mark();
  if (S->precond) {
    launch_degrid_dual_precond(op, 0, L, S->v2.p, S->gold.p, S->y.p, S->projw.p, s, true);
    mark();
    launch_block_reduce_precond(op, 0, L, s);
    mark();
    launch_fb_iterations(op, 0, L, S->projw.p, S->y.p, S->fb_max, S->fb_min, S->fb_stop, s);
    mark();
    launch_grid_dual_precond(op, 0, L, S->v2.p, S->projw.p, s);
    mark();
  } else {
    launch_degrid_dual(op, 0, L, S->v2.p, S->gold.p, S->y.p, s, true);
    mark();
    launch_block_reduce(op, 0, L, s);
    mark();
    mark();
    launch_grid_dual(op, 0, L, S->v2.p, s);
    mark();
  }
  solver_fft_inverse(op, s);
  mark();
  FHS_CUDA(cudaMemsetAsync(S->l21_acc.p, 0, S->G * sizeof(double), s));
  if (sara_fused_supported(S->lg)) {
    sara_analysis_prox(S->sp, S->xhat.p, S->v1.p, S->apx.p, S->w1.p, S->beta1.p, S->G, S->lg, S->l21_acc.p, s);
    mark();
  } else {
    sara_analysis(S->sp, S->xhat.p, S->coef.p, S->apx.p, L, s);
    mark();
    sara_l21_prox(S->sp, S->v1.p, S->coef.p, S->xhat.p, S->w1.p, S->beta1.p, S->G, S->lg, S->l21_part.p, s);
  }
  mark();
  sara_synthesis(S->sp, S->v1.p, S->g1.p, S->apx.p, L, (float)S->sigma11, s);
  mark();
  if (S->nuclear) nuc_gram(S->np, S->xhat.p, S->v0.p, s);
  mark();
  if (S->nuclear) nuc_eig(S->np, S->w0.p, S->beta0.p, S->nuc_vals.p, s);
  mark();
  if (S->nuclear) nuc_reconstruct(S->np, S->xhat.p, S->v0.p, s);
  mark();
  AssembleArgs a;
  a.Ny = S->Ny;
  a.Nx = S->Nx;
  a.Ky = op->Ky;
  a.Kx = op->Kx;
  a.lg = S->lg;
  a.Qy = S->nuclear ? S->np.Qy : 1;
  a.nuclear = S->nuclear ? 1 : 0;
  a.img_compact = op->own_fft ? 1 : 0;
  a.sigma00 = (float)S->sigma00;
  a.facets = S->nuclear ? S->np.d_facets.p : nullptr;
  a.wy = S->nuclear ? S->np.wy.p : nullptr;
  a.wx = S->nuclear ? S->np.wx.p : nullptr;
  a.cover_y = S->nuclear ? S->np.cover_y.p : nullptr;
  a.cover_x = S->nuclear ? S->np.cover_x.p : nullptr;
  a.v0_group = S->nuclear ? S->np.v0_group : 0;
  assemble_kernel<<<nblk(S->N), 256, 0, s>>>(a, L, S->g.p, op->imgr.p, S->g1.p, S->v0.p, S->sigma22.p,
                                           op->sy.p, op->sx.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  mark();
  stats_kernel<<<S->G, 256, 0, s>>>(S->primal_part.p, kPrimalBlocks, S->lg, S->G, op->blk_stats.p, op->ch_nblk.p,
                                op->ch_blkoff.p, op->blk_eps.p, S->nuclear ? S->nuc_vals.p : nullptr,
                                S->nuclear ? S->np.Q : 0, S->l21_part.p,
                                sara_fused_supported(S->lg) ? 0 : S->prox_blocks, S->l21_acc.p, S->ring.p,
                                S->ring_counter.p, S->ring_counter.p + 1);
  count_launch();
  FHS_LAUNCH_CHECK();
  mark();
}

static void solver_capture(Solver* S) {
  cudaStream_t s = S->op->stream;
  S->graph_epoch = S->op->layout_epoch;
  if (S->graph) {
    cudaGraphExecDestroy(S->graph);
    S->graph = nullptr;
  }
  const unsigned long long before = g_launches;
  cudaGraph_t g = nullptr;
  FHS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    solver_launch_iteration(S, s);
  } catch (...) {
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  FHS_CUDA(cudaStreamEndCapture(s, &g));
  cudaError_t e = cudaGraphInstantiate(&S->graph, g, 0);
  cudaGraphDestroy(g);
  FHS_CUDA(e);
  S->launches_per_iter = g_launches - before;
  g_launches = before;
}

// weights1 from ||Psit x||_row and weights0 from the facet singular values
// (fhs_update_weights.m:73-92, sara.m:764-768).
static void solver_update_weights(Solver* S) {
  cudaStream_t s = S->op->stream;
  sara_analysis(S->sp, S->x.p, S->coef.p, S->apx.p, S->L, s);
  sara_row_norms(S->sp, S->coef.p, S->x.p, S->G, S->lg, S->rownorm.p, s);
  weights_kernel<<<dim3(nblk(S->sp.s), S->G), 256, 0, s>>>(S->rownorm.p, S->sp.s, S->sig.p, S->w1.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  if (S->nuclear) {
    nuc_gram(S->np, S->x.p, nullptr, s);
    nuc_eig(S->np, nullptr, nullptr, nullptr, s);
    weights0_kernel<<<S->G * S->np.Q, 64, 0, s>>>(S->np.sigma.p, S->lg, S->sig_bar.p, S->w0.p);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
}

}  // namespace fhs

using namespace fhs;

namespace fhs {
template <class F>
fhs_status guarded_solver(F&& f) {
  try {
    f();
    set_last_error("");
    return FHS_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return FHS_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FHS_ERR_INVALID_ARG;
  }
}
static Solver* sv(fhs_solver* s) {
  FHS_CHECK(s != nullptr, FHS_ERR_INVALID_ARG, "null solver handle");
  return reinterpret_cast<Solver*>(s);
}
}  // namespace fhs

extern "C" {

fhs_status fhs_solver_create(fhs_measop* op_, const fhs_solver_config* cfg, fhs_solver** out) {
  return guarded_solver([&] {
    FHS_CHECK(op_ && cfg && out, FHS_ERR_INVALID_ARG, "null argument");
    MeasOp* op = reinterpret_cast<MeasOp*>(op_);
    FHS_CHECK(op->committed, FHS_ERR_STATE, "operator not committed");
    FHS_CHECK(cfg->algo >= FHS_ALGO_SARA && cfg->algo <= FHS_ALGO_FHS, FHS_ERR_INVALID_ARG, "bad algo");
    DeviceGuard dg(op->device);
    cudaStream_t s = op->stream;
    auto S = std::make_unique<Solver>();
    S->op = op;
    S->device = op->device;
    S->algo = cfg->algo;
    S->nlevel = cfg->nlevel > 0 ? cfg->nlevel : 4;
    S->L = op->L;
    S->Ny = op->Ny;
    S->Nx = op->Nx;
    S->N = op->Npix();
    if (S->algo == FHS_ALGO_SARA) {
      S->G = S->L;
      S->lg = 1;
      S->nuclear = false;
    } else {
      S->G = cfg->n_groups > 0 ? cfg->n_groups : 1;
      FHS_CHECK(S->L % S->G == 0, FHS_ERR_INVALID_ARG, "channels must split evenly into groups");
      S->lg = S->L / S->G;
      S->nuclear = true;
    }
    S->sp = sara_plan(S->Ny, S->Nx, S->nlevel);
    measop_enable_r2c(op);
    if (S->nuclear) {
      int Qy = 1, Qx = 1, oy = 0, ox = 0, win = FHS_WINDOW_NONE;
      std::vector<int> sy, sx;
      if (S->algo == FHS_ALGO_FHS) {
        Qy = std::max(cfg->Qy, 1);
        Qx = std::max(cfg->Qx, 1);
        oy = std::max(cfg->overlap_y, 0);
        ox = std::max(cfg->overlap_x, 0);
        win = cfg->window;
      }
      auto splits = [](const int* given, int Q, int N) {
        std::vector<int> v(Q + 1);
        for (int q = 0; q <= Q; ++q)
          v[q] = given ? given[q] : (int)std::floor((double)q * N / Q + 0.5);  // split_range
        return v;
      };
      sy = splits(S->algo == FHS_ALGO_FHS ? cfg->splits_y : nullptr, Qy, S->Ny);
      sx = splits(S->algo == FHS_ALGO_FHS ? cfg->splits_x : nullptr, Qx, S->Nx);
      nuc_plan_init(S->np, S->Ny, S->Nx, Qy, Qx, sy, sx, oy, ox, win, S->G, S->lg, s);
    }
    const int64_t L = S->L, N = S->N, sc = S->sp.s;
    S->x.alloc(L * N);
    S->g.alloc(L * N);
    S->xhat.alloc(L * N);
    S->g1.alloc(L * N);
    S->coef.alloc(L * sc);  // analysis output for weights (and the unfused prox path)
    S->apx.alloc(L * S->sp.apx_total);
    S->v1.alloc(L * sc);
    S->w1.alloc((size_t)S->G * sc);
    S->rownorm.alloc((size_t)S->G * sc);
    S->beta1.alloc(S->G);
    S->sig.alloc(S->G);
    if (S->nuclear) {
      S->v0.alloc((size_t)S->G * S->np.v0_group);
      S->w0.alloc((size_t)S->G * S->np.Q * S->lg);
      S->beta0.alloc((size_t)S->G * S->np.Q);
      S->sig_bar.alloc((size_t)S->G * S->np.Q);
      S->nuc_vals.alloc((size_t)S->G * S->np.Q);
    }
    S->y.alloc(std::max<int64_t>(op->Mtot, 1));
    S->y.zero(s);
    S->v2.alloc(std::max<int64_t>(op->Mtot, 1));
    S->gold.alloc(std::max<int64_t>(op->Mtot, 1));
    S->sigma22.alloc(L);
    S->primal_part.alloc(L * kPrimalBlocks * 2);
    S->prox_blocks = nblk(sc);
    S->l21_part.alloc((size_t)S->G * S->prox_blocks);
    S->l21_acc.alloc(S->G);
    S->l21_acc.zero(s);
    S->ring.alloc((size_t)kReportRing * S->G * kReportFields);
    S->ring_counter.alloc(2);  // [0] iterations recorded, [1] CTAs done in the current one
    S->ring_counter.zero(s);
    FHS_CUDA(cudaStreamSynchronize(s));
    *out = reinterpret_cast<fhs_solver*>(S.release());
  });
}

fhs_status fhs_solver_destroy(fhs_solver* s) {
  return guarded_solver([&] {
    Solver* S = reinterpret_cast<Solver*>(s);
    if (!S) return;
    DeviceGuard dg(S->device);
    delete S;
  });
}

fhs_status fhs_solver_set_data(fhs_solver* s_, const double* y, const double* eps) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(y && eps, FHS_ERR_INVALID_ARG, "null buffer");
    MeasOp* op = S->op;
    DeviceGuard dg(op->device);
    cudaStream_t s = op->stream;
    if (op->stage.n < (size_t)2 * op->Mtot) op->stage.alloc(2 * std::max<int64_t>(op->Mtot, 1));
    FHS_CUDA(cudaMemcpyAsync(op->stage.p, y, 2 * op->Mtot * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_vis_gather(op->stage.p, S->y.p, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, op->L, op->maxM, 0, s);
    std::vector<double> e((size_t)op->L * kMaxBlocksPerChannel, 0.0);
    for (int l = 0; l < op->L; ++l)
      for (int b = 0; b < op->h_nblk[l]; ++b) {
        const double v = eps[op->h_blkoff[l] + b];
        FHS_CHECK(std::isfinite(v) && v >= 0, FHS_ERR_INVALID_ARG, "epsilon must be finite and >= 0");
        e[(size_t)l * kMaxBlocksPerChannel + b] = v;
      }
    op->blk_eps.upload(e.data(), e.size(), s);
    S->h_eps.assign(eps, eps + op->nblk_tot);
    FHS_CUDA(cudaStreamSynchronize(s));
    S->data_set = true;
  });
}

fhs_status fhs_solver_set_params(fhs_solver* s_, const fhs_solver_params* p) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(p && p->nu2 && p->gamma && p->reweighting_sig, FHS_ERR_INVALID_ARG, "null parameter array");
    FHS_CHECK(!S->nuclear || (p->gamma0 && p->reweighting_sig_bar), FHS_ERR_INVALID_ARG,
              "gamma0 and reweighting_sig_bar are required");
    FHS_CHECK(p->nu0 > 0 && p->nu1 > 0, FHS_ERR_INVALID_ARG, "nu0 and nu1 must be > 0");
    DeviceGuard dg(S->op->device);
    cudaStream_t s = S->op->stream;
    const int G = S->G, Q = S->nuclear ? S->np.Q : 0;
    S->nu2.assign(p->nu2, p->nu2 + S->L);
    for (double v : S->nu2) FHS_CHECK(v > 0 && std::isfinite(v), FHS_ERR_INVALID_ARG, "nu2 must be > 0");
    S->gamma.assign(p->gamma, p->gamma + G);
    S->rw_sig.assign(p->reweighting_sig, p->reweighting_sig + G);
    if (S->nuclear) {
      S->gamma0.assign(p->gamma0, p->gamma0 + (size_t)G * Q);
      S->rw_sig_bar.assign(p->reweighting_sig_bar, p->reweighting_sig_bar + (size_t)G * Q);
    }
    S->rw_alpha = p->reweighting_alpha;
    S->rw_flag = p->reweighting_flag;
    S->rw_min = p->reweighting_min_iter;
    S->rw_max = p->reweighting_max_iter;
    S->rw_rel_var = p->reweighting_rel_var;
    S->pdfb_min = p->pdfb_min_iter;
    S->pdfb_max = p->pdfb_max_iter;
    S->pdfb_rel_var = p->pdfb_rel_var;
    S->pdfb_tol = p->pdfb_fidelity_tolerance;
    S->pdfb_rel_var_low = p->pdfb_rel_var_low;
    if (p->elipse_proj_max_iter > 0) {
      FHS_CHECK(p->elipse_proj_min_iter >= 0 && p->elipse_proj_eps >= 0, FHS_ERR_INVALID_ARG,
                "bad ellipsoid-projection parameters");
      S->fb_max = p->elipse_proj_max_iter;
      S->fb_min = p->elipse_proj_min_iter;
      S->fb_stop = p->elipse_proj_eps;
    } else {  // imaging/default_parameters.json "proj"
      S->fb_max = 20;
      S->fb_min = 1;
      S->fb_stop = 1e-8;
    }
    S->adjust_noise = p->adjust_flag_noise != 0 && S->algo != FHS_ALGO_SARA;
    S->adjust_min_iter = p->adjust_noise_min_iter > 0 ? p->adjust_noise_min_iter : 100;
    S->adjust_rel_var = p->adjust_noise_rel_var > 0 ? p->adjust_noise_rel_var : 1e-3;
    S->adjust_start_iter = p->adjust_noise_start_iter > 0 ? p->adjust_noise_start_iter : 2000;
    S->adjust_change = p->adjust_noise_change_percentage > 0 ? p->adjust_noise_change_percentage : 0.5;
    S->alph = p->alph > 0 ? p->alph : 1.0;
    S->alph_bar = p->alph_bar > 0 ? p->alph_bar : 1.0;
    const double sigma0 = 1.0 / p->nu0, sigma1 = 1.0 / p->nu1;
    S->sigma0 = sigma0;
    S->sigma1 = sigma1;
    // facetHyperSARA.m:582-608 / hyperSARA.m:471-487: tau = 0.99/3;
    // sara.m:502-505: tau = 0.99/(sigma1 nu1 + sigma2 nu2) = 0.99/2
    S->tau = S->algo == FHS_ALGO_SARA ? 0.99 / 2.0 : 0.99 / 3.0;
    S->sigma00 = S->tau * sigma0;
    S->sigma11 = S->tau * sigma1;
    std::vector<float> s22(S->L);
    for (int l = 0; l < S->L; ++l) s22[l] = (float)(S->tau / S->nu2[l]);
    S->sigma22.upload(s22.data(), S->L, s);
    std::vector<double> b1(G), ups(G);
    for (int g = 0; g < G; ++g) {
      b1[g] = S->gamma[g] / sigma1;
      ups[g] = S->rw_sig[g] * S->rw_alpha;
    }
    S->beta1.upload(b1.data(), G, s);
    S->sig.upload(ups.data(), G, s);
    if (S->nuclear) {
      std::vector<double> b0((size_t)G * Q), ub((size_t)G * Q);
      for (size_t i = 0; i < b0.size(); ++i) {
        b0[i] = S->gamma0[i] / sigma0;
        ub[i] = S->rw_sig_bar[i] * S->rw_alpha;
      }
      S->beta0.upload(b0.data(), b0.size(), s);
      S->sig_bar.upload(ub.data(), ub.size(), s);
    }
    FHS_CUDA(cudaStreamSynchronize(s));
    S->params_set = true;
  });
}

}  // extern "C"

namespace fhs {

void solver_init_state(Solver* S, const double* xinit, const float* xinit_dev) {
  FHS_CHECK(S->params_set && S->data_set, FHS_ERR_STATE, "set data and params before init");
  MeasOp* op = S->op;
  DeviceGuard dg(op->device);
  cudaStream_t s = op->stream;
  if (!op->tuned) measop_autotune(op);   // before any state: the timed launches use scratch only
  const int64_t n = (int64_t)S->L * S->N;
  if (xinit) {
    if (op->stage.n < (size_t)n) op->stage.alloc(n);
    FHS_CUDA(cudaMemcpyAsync(op->stage.p, xinit, n * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_d2f(op->stage.p, S->x.p, n, s);
  } else if (xinit_dev) {
    FHS_CUDA(cudaMemcpyAsync(S->x.p, xinit_dev, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  } else {
    S->x.zero(s);
  }
  S->g.zero(s);
  S->v1.zero(s);
  S->v2.zero(s);
  S->g1.zero(s);
  if (S->nuclear) S->v0.zero(s);
  S->ring_counter.zero(s);
  // Fx_old: keep G A x_init per visibility (linearity of G)
  if (!op->own_fft) launch_pad_real(op, S->x.p, 0, S->L, s);
  solver_fft_forward(op, S->x.p, s);
  launch_degrid_plain(op, 0, S->L, S->gold.p, s, true);
  S->precond = op->precond;
  if (S->precond) {
    if (S->projw.n < (size_t)std::max<int64_t>(op->Mtot, 1)) S->projw.alloc(std::max<int64_t>(op->Mtot, 1));
    launch_w_from_proj(op, nullptr, S->y.p, S->projw.p, s);  // proj = 0 (fhs_initialize_data_worker.m:43)
    if (S->algo == FHS_ALGO_SARA) {
      // sara.m:420-428: proj starts as the projection of G A x0 from zero.
      // With v2 = 0 and gold = G A x0 the dual pass 1 gives d = G A x0 - y.
      launch_degrid_dual_precond(op, 0, S->L, S->v2.p, S->gold.p, S->y.p, S->projw.p, s, true);
      launch_block_reduce_precond(op, 0, S->L, s);
      launch_fb_iterations(op, 0, S->L, S->projw.p, S->y.p, S->fb_max, S->fb_min, S->fb_stop, s);
    }
  }
  solver_update_weights(S);
  FHS_CUDA(cudaStreamSynchronize(s));
  solver_capture(S);
  S->iter_done = 0;
  S->ring_read = 0;
  S->initialised = true;
}

}  // namespace fhs

extern "C" {

fhs_status fhs_solver_init(fhs_solver* s_, const double* xinit) {
  return guarded_solver([&] { solver_init_state(sv(s_), xinit, nullptr); });
}

// the iteration graph holds the operator's work lists and launch shapes:
// capture it again after the autotuner or fhs_measop_set_tuning changed them
static void ensure_graph(Solver* S) {
  if (S->graph_epoch != S->op->layout_epoch) solver_capture(S);
}

static void read_ring(Solver* S, long long first, int n, std::vector<double>& rec) {
  cudaStream_t s = S->op->stream;
  const size_t per = (size_t)S->G * kReportFields;
  rec.resize((size_t)n * per);
  for (int i = 0; i < n; ++i) {
    const long long slot = (first + i) % kReportRing;
    FHS_CUDA(cudaMemcpyAsync(rec.data() + i * per, S->ring.p + slot * per, per * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
  }
  FHS_CUDA(cudaStreamSynchronize(s));
}

static void fill_info(const Solver* S, const double* rec, fhs_iter_info* info) {
  double rx = 0, nx = 0, r2 = 0, e2 = 0, nu = 0;
  for (int g = 0; g < S->G; ++g) {
    rx += rec[g * kReportFields + 0];
    nx += rec[g * kReportFields + 1];
    r2 += rec[g * kReportFields + 2];
    e2 += rec[g * kReportFields + 3];
    nu += rec[g * kReportFields + 4];
  }
  info->rel_val = nx > 0 ? std::sqrt(rx / nx) : 0.0;
  info->residual = std::sqrt(r2);
  info->epsilon = std::sqrt(e2);
  info->nuclear = nu;
}

fhs_status fhs_solver_iterate(fhs_solver* s_, int n, fhs_iter_info* info) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    FHS_CHECK(n >= 0, FHS_ERR_INVALID_ARG, "negative iteration count");
    DeviceGuard dg(S->op->device);
    cudaStream_t s = S->op->stream;
    ensure_graph(S);
    int done = 0;
    std::vector<double> rec;
    while (done < n) {
      const int chunk = std::min(n - done, kReportRing);
      for (int i = 0; i < chunk; ++i) FHS_CUDA(cudaGraphLaunch(S->graph, s));
      g_launches += S->launches_per_iter * chunk;
      if (info) {
        read_ring(S, S->iter_done, chunk, rec);
        for (int i = 0; i < chunk; ++i) fill_info(S, rec.data() + (size_t)i * S->G * kReportFields, info + done + i);
      }
      S->iter_done += chunk;
      done += chunk;
    }
    if (!info) FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_solver_group_stats(fhs_solver* s_, double* out) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null output");
    FHS_CHECK(S->iter_done >= 1, FHS_ERR_STATE, "no iteration run since fhs_solver_init");
    DeviceGuard dg(S->op->device);
    std::vector<double> rec;
    read_ring(S, S->iter_done - 1, 1, rec);
    for (int g = 0; g < S->G; ++g)
      for (int f = 0; f < 4; ++f) out[g * 4 + f] = rec[(size_t)g * kReportFields + f];
  });
}

fhs_status fhs_solver_update_weights(fhs_solver* s_) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    DeviceGuard dg(S->op->device);
    solver_update_weights(S);
    FHS_CUDA(cudaStreamSynchronize(S->op->stream));
  });
}

// beta1 = gamma / sigma1, beta0 = gamma0 / sigma0 from the host copies (or 0:
// priors off, facetHyperSARA.m:704-708)
static void upload_betas(Solver* S, bool off) {
  cudaStream_t s = S->op->stream;
  const int G = S->G;
  std::vector<double> b1(G);
  for (int g = 0; g < G; ++g) b1[g] = off ? 0.0 : S->gamma[g] / S->sigma1;
  S->beta1.upload(b1.data(), G, s);
  if (S->nuclear) {
    std::vector<double> b0(S->gamma0.size());
    for (size_t i = 0; i < b0.size(); ++i) b0[i] = off ? 0.0 : S->gamma0[i] / S->sigma0;
    S->beta0.upload(b0.data(), b0.size(), s);
  }
  FHS_CUDA(cudaStreamSynchronize(s));
}

// facetHyperSARA.m:903-937 / hyperSARA.m:697-731: adapts the l2 bounds from
// the last block residuals, re-estimates the channel noise levels and sets
// gamma / gamma0 from compute_noise_level.m:49-89 (FP64, host).
static void adjust_noise_level(Solver* S) {
  MeasOp* op = S->op;
  cudaStream_t s = op->stream;
  std::vector<double> st((size_t)op->nblk_tot * 2);
  op->blk_stats.download(st.data(), st.size(), s);
  FHS_CUDA(cudaStreamSynchronize(s));
  std::vector<double> e((size_t)op->L * kMaxBlocksPerChannel, 0.0), sig_ch(op->L, 0.0);
  for (int l = 0; l < op->L; ++l) {
    double e2 = 0.0, m = 0.0;
    for (int b = 0; b < op->h_nblk[l]; ++b) {
      const int gb = op->h_blkoff[l] + b;
      const double r = std::sqrt(st[2 * gb + 1]);
      double& eps = S->h_eps[gb];
      if (eps < (2.0 - S->pdfb_tol) * r) eps = (eps + r) * S->adjust_change;
      e[(size_t)l * kMaxBlocksPerChannel + b] = eps;
      e2 += eps * eps;
      m += (double)op->ch[l].block_sizes[b];
    }
    // expectation of std() of the reference's randn draw with per-block
    // variance eps_b^2 / M_b
    sig_ch[l] = m > 0 ? std::sqrt(e2 / m) : 0.0;
  }
  op->blk_eps.upload(e.data(), e.size(), s);
  const int lg = S->lg;
  const double mu_chi = std::sqrt(2.0) * std::exp(std::lgamma((lg + 1) / 2.0) - std::lgamma(lg / 2.0));
  const double sig_chi = std::sqrt(std::max(lg - mu_chi * mu_chi, 0.0));
  for (int g = 0; g < S->G; ++g) {
    double ssum = 0.0;
    for (int i = 0; i < lg; ++i) {
      const int l = g * lg + i;
      if (S->nu2[l] > 0) ssum += sig_ch[l] * sig_ch[l] / S->nu2[l];  // a channel without data adds nothing
    }
    const double sig_sara = std::sqrt(ssum / lg);
    S->gamma[g] = S->alph * sig_sara * (mu_chi + sig_chi);
    if (S->nuclear) {
      for (int q = 0; q < S->np.Q; ++q) {
        const NucFacet& f = S->np.facets[q];
        const double P = (double)(f.y1 - f.y0) * (double)(f.x1 - f.x0);
        S->gamma0[(size_t)g * S->np.Q + q] = S->alph_bar * std::sqrt(P * ssum / std::min(P, (double)lg));
      }
    }
  }
  upload_betas(S, false);
}

fhs_status fhs_solver_run(fhs_solver* s_, int max_iter, fhs_run_info* out) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    DeviceGuard dg(S->op->device);
    cudaStream_t s = S->op->stream;
    const auto t0 = std::chrono::steady_clock::now();
    if (max_iter <= 0) max_iter = (S->rw_max + 1) * S->pdfb_max;
    const int64_t n = (int64_t)S->L * S->N;
    DevBuf<float> x_rw;
    x_rw.alloc(n);
    FHS_CUDA(cudaMemcpyAsync(x_rw.p, S->x.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    DevBuf<double> dn;
    const int nb = nblk(n);
    dn.alloc(2 * nb);
    std::vector<double> hdn(2 * nb), rec;
    int last = 0, rw_count = 0, t = 0, converged = 0, n_adjust = 0;
    fhs_iter_info info{};
    bool adjust = S->adjust_noise;
    if (adjust) upload_betas(S, true);  // priors off until the first adjustment
    ensure_graph(S);
    // The stopping statistics stay in the device ring until a test needs
    // them: while t - last < pdfb_min_iter (and no noise adjustment is
    // pending) the PDFB test cannot fire, so the graphs are launched back to
    // back and their records read together at the next test.
    int pending = 0;
    for (t = 1; t <= max_iter; ++t) {
      FHS_CUDA(cudaGraphLaunch(S->graph, s));
      g_launches += S->launches_per_iter;
      S->iter_done += 1;
      ++pending;
      if (!adjust && t - last < S->pdfb_min && t < max_iter && pending < kReportRing / 2) continue;
      read_ring(S, S->iter_done - pending, pending, rec);
      for (int i = 0; i < pending; ++i) {
        fill_info(S, rec.data() + (size_t)i * S->G * kReportFields, &info);
        FHS_CHECK(std::isfinite(info.rel_val) && std::isfinite(info.residual), FHS_ERR_NUMERIC,
                  "non-finite iterate at iteration " + std::to_string(t - pending + 1 + i));
      }
      pending = 0;
      const bool pdfb = (t - last >= S->pdfb_min) &&
                        (t - last >= S->pdfb_max ||
                         (info.rel_val <= S->pdfb_rel_var && info.residual <= S->pdfb_tol * info.epsilon) ||
                         info.rel_val <= S->pdfb_rel_var_low);
      if (adjust && info.residual > S->pdfb_tol * info.epsilon) {
        // facetHyperSARA.m:883-889 (also at the run's first iteration) /
        // hyperSARA.m:690-695 (at adjust_noise_start_iter instead)
        const bool early = S->algo == FHS_ALGO_FHS ? last < 1 : (last < 1 && t == S->adjust_start_iter);
        if (t - last >= S->pdfb_max || early ||
            (info.rel_val <= S->adjust_rel_var && t - last >= S->adjust_min_iter)) {
          adjust_noise_level(S);
          ++n_adjust;
          last = t;
          continue;
        }
      }
      if (!pdfb) continue;
      adjust = false;  // facetHyperSARA.m:952
      diff_norm_kernel<<<nb, 256, 0, s>>>(x_rw.p, S->x.p, n, dn.p);
      count_launch();
      FHS_LAUNCH_CHECK();
      dn.download(hdn.data(), 2 * nb, s);
      FHS_CUDA(cudaStreamSynchronize(s));
      double d2 = 0, a2 = 0;
      for (int i = 0; i < nb; ++i) {
        d2 += hdn[2 * i];
        a2 += hdn[2 * i + 1];
      }
      const double rel_rw = std::sqrt(d2 / std::max(a2, 1e-300));
      if (!S->rw_flag || (rw_count >= S->rw_min && (rw_count >= S->rw_max || rel_rw <= S->rw_rel_var))) {
        converged = 1;
        break;
      }
      solver_update_weights(S);
      FHS_CUDA(cudaMemcpyAsync(x_rw.p, S->x.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
      ++rw_count;
      last = t;
    }
    FHS_CUDA(cudaStreamSynchronize(s));
    if (out) {
      out->n_iter = std::min(t, max_iter);
      out->n_reweights = rw_count;
      out->converged = converged;
      out->rel_val = info.rel_val;
      out->residual = info.residual;
      out->epsilon = info.epsilon;
      out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      out->n_noise_adjustments = n_adjust;
    }
  });
}

fhs_status fhs_solver_ellipse_iterations(fhs_solver* s_, int* counts) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(counts != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    MeasOp* op = S->op;
    std::vector<int> c((size_t)op->L * kMaxBlocksPerChannel, 0);
    if (S->precond) {
      DeviceGuard dg(op->device);
      op->fb_count.download(c.data(), c.size(), op->stream);
      FHS_CUDA(cudaStreamSynchronize(op->stream));
    }
    for (int l = 0; l < op->L; ++l)
      for (int b = 0; b < op->h_nblk[l]; ++b) counts[op->h_blkoff[l] + b] = c[(size_t)l * kMaxBlocksPerChannel + b];
  });
}

fhs_status fhs_solver_epsilon(fhs_solver* s_, double* epsilon) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(epsilon != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    FHS_CHECK(S->data_set, FHS_ERR_STATE, "no data set");
    std::copy(S->h_eps.begin(), S->h_eps.end(), epsilon);
  });
}

fhs_status fhs_solver_set_epsilon(fhs_solver* s_, const double* epsilon) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(epsilon != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    FHS_CHECK(S->data_set, FHS_ERR_STATE, "set data first");
    MeasOp* op = S->op;
    DeviceGuard dg(op->device);
    std::vector<double> e((size_t)op->L * kMaxBlocksPerChannel, 0.0);
    for (int l = 0; l < op->L; ++l)
      for (int b = 0; b < op->h_nblk[l]; ++b) {
        const double v = epsilon[op->h_blkoff[l] + b];
        FHS_CHECK(std::isfinite(v) && v >= 0, FHS_ERR_INVALID_ARG, "epsilon must be finite and >= 0");
        e[(size_t)l * kMaxBlocksPerChannel + b] = v;
      }
    op->blk_eps.upload(e.data(), e.size(), op->stream);
    S->h_eps.assign(epsilon, epsilon + op->nblk_tot);
    FHS_CUDA(cudaStreamSynchronize(op->stream));
  });
}

fhs_status fhs_solver_regularization(fhs_solver* s_, double* gamma, double* gamma0) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(gamma != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    FHS_CHECK(S->params_set, FHS_ERR_STATE, "no parameters set");
    std::copy(S->gamma.begin(), S->gamma.end(), gamma);
    if (gamma0 && S->nuclear) std::copy(S->gamma0.begin(), S->gamma0.end(), gamma0);
  });
}

}  // extern "C"

namespace fhs {
namespace {

// Number of doubles of one state field in the host layout (0: not present).
int64_t field_size(const Solver* S, int field) {
  const MeasOp* op = S->op;
  const int64_t LN = (int64_t)S->L * S->N;
  switch (field) {
    case FHS_FIELD_X:
    case FHS_FIELD_G:
      return LN;
    case FHS_FIELD_V0:
      return S->nuclear ? (int64_t)S->G * S->np.v0_group : 0;
    case FHS_FIELD_V1:
      return (int64_t)S->L * S->sp.s;
    case FHS_FIELD_V2:
      return 2 * op->Mtot;
    case FHS_FIELD_PROJ:
      return S->precond ? 2 * op->Mtot : 0;
    case FHS_FIELD_WEIGHTS0:
      return S->nuclear ? (int64_t)S->G * S->np.Q * S->lg : 0;
    case FHS_FIELD_WEIGHTS1:
      return (int64_t)S->G * S->sp.s;
    default:
      return -1;
  }
}

float* float_field(Solver* S, int field) {
  switch (field) {
    case FHS_FIELD_X: return S->x.p;
    case FHS_FIELD_G: return S->g.p;
    case FHS_FIELD_V0: return S->v0.p;
    case FHS_FIELD_V1: return S->v1.p;
    case FHS_FIELD_WEIGHTS1: return S->w1.p;
    default: return nullptr;
  }
}

void state_io(Solver* S, int field, double* out, const double* in) {
  FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
  const int64_t n = field_size(S, field);
  FHS_CHECK(n >= 0, FHS_ERR_INVALID_ARG, "unknown state field");
  if (n == 0) return;
  FHS_CHECK(out || in, FHS_ERR_INVALID_ARG, "null buffer");
  MeasOp* op = S->op;
  DeviceGuard dg(op->device);
  cudaStream_t s = op->stream;
  if (op->stage.n < (size_t)n) op->stage.alloc(n);
  double* st = op->stage.p;
  if (in) FHS_CUDA(cudaMemcpyAsync(st, in, n * sizeof(double), cudaMemcpyHostToDevice, s));
  switch (field) {
    case FHS_FIELD_V2:
      if (in)
        launch_vis_gather(st, S->v2.p, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, op->L, op->maxM, 0, s);
      else
        launch_vis_scatter(S->v2.p, st, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, op->L, op->maxM, 0, s);
      break;
    case FHS_FIELD_PROJ:
      if (in)
        launch_w_from_proj(op, st, S->y.p, S->projw.p, s);
      else
        launch_proj_from_w(op, S->projw.p, S->y.p, st, s);
      break;
    case FHS_FIELD_WEIGHTS0:
      if (in)
        FHS_CUDA(cudaMemcpyAsync(S->w0.p, st, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      else
        FHS_CUDA(cudaMemcpyAsync(st, S->w0.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      break;
    default:
      if (in)
        launch_d2f(st, float_field(S, field), n, s);
      else
        launch_f2d(float_field(S, field), st, n, s);
  }
  if (out) FHS_CUDA(cudaMemcpyAsync(out, st, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace fhs

extern "C" {

int64_t fhs_solver_field_size(const fhs_solver* s_, int field) {
  const Solver* S = reinterpret_cast<const Solver*>(s_);
  if (!S) return -1;
  return field_size(S, field);
}

fhs_status fhs_solver_get_field(fhs_solver* s_, int field, double* out) {
  return guarded_solver([&] {
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    state_io(sv(s_), field, out, nullptr);
  });
}

fhs_status fhs_solver_set_field(fhs_solver* s_, int field, const double* in) {
  return guarded_solver([&] {
    FHS_CHECK(in != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    state_io(sv(s_), field, nullptr, in);
  });
}

int fhs_solver_stage_count(void) { return kStages; }

const char* fhs_solver_stage_name(int i) { return (i >= 0 && i < kStages) ? kStageNames[i] : ""; }

fhs_status fhs_solver_time_iterations(fhs_solver* s_, int n, double* ms) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    FHS_CHECK(n > 0 && ms, FHS_ERR_INVALID_ARG, "bad arguments");
    DeviceGuard dg(S->op->device);
    cudaStream_t s = S->op->stream;
    cudaEvent_t e0, e1;
    FHS_CUDA(cudaEventCreate(&e0));
    FHS_CUDA(cudaEventCreate(&e1));
    ensure_graph(S);
    FHS_CUDA(cudaStreamSynchronize(s));
    FHS_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < n; ++i) FHS_CUDA(cudaGraphLaunch(S->graph, s));
    FHS_CUDA(cudaEventRecord(e1, s));
    FHS_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    FHS_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g_launches += S->launches_per_iter * n;
    S->iter_done += n;
    *ms = t;
  });
}

fhs_status fhs_solver_profile_stages(fhs_solver* s_, int n, double* stage_ms) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(S->initialised, FHS_ERR_STATE, "solver not initialised");
    FHS_CHECK(n > 0 && stage_ms, FHS_ERR_INVALID_ARG, "bad arguments");
    DeviceGuard dg(S->op->device);
    cudaStream_t s = S->op->stream;
    cudaEvent_t ev[kStages + 1];
    for (auto& e : ev) FHS_CUDA(cudaEventCreate(&e));
    std::vector<double> acc(kStages, 0.0);
    for (int it = 0; it < n; ++it) {
      solver_launch_iteration(S, s, ev);
      FHS_CUDA(cudaEventSynchronize(ev[kStages]));
      for (int k = 0; k < kStages; ++k) {
        float t = 0.f;
        FHS_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
        acc[k] += t;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    S->iter_done += n;
    for (int k = 0; k < kStages; ++k) stage_ms[k] = acc[k] / n;
  });
}

fhs_status fhs_solver_get_x(fhs_solver* s_, double* x) {
  return guarded_solver([&] {
    Solver* S = sv(s_);
    FHS_CHECK(x != nullptr, FHS_ERR_INVALID_ARG, "null buffer");
    MeasOp* op = S->op;
    DeviceGuard dg(op->device);
    cudaStream_t s = op->stream;
    const int64_t n = (int64_t)S->L * S->N;
    if (op->stage.n < (size_t)n) op->stage.alloc(n);
    launch_f2d(S->x.p, op->stage.p, n, s);
    FHS_CUDA(cudaMemcpyAsync(x, op->stage.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
