// Learned warm start on the device: dirty cube -> network -> fallback rule
// -> solver initialisation, without a host round trip of any cube.
//
// The solvers take an initial estimate x0 (the xinit / varargin{1} of
// src/fhs/facetHyperSARA.m:1-6, used at :347-350).  This entry point forms
// it from the solver's own data:
//  * the normalised dirty cube Re(Phi^H y) / PSF peak per channel
//    (src/compute_residual_images.m:83-102 at x = 0), Phi = G A of the
//    solver's operator, y its whitened visibilities;
//  * the warm-start network on every channel (images [Nx][Ny], the solver's
//    plane layout), clipped at 0 as the primal update clips
//    (fhs_update_primal.m:33-38);
//  * the objective F(x) = sum_b max(0, ||y_b - Phi_b x|| - eps_b)
//    + sum_g gamma_g ||Psi^T x_g||_{2,1} + sum_g gamma0_g ||x_g||_* (nuclear
//    term for the FHS / HS priors, taken over each whole sub-cube with the
//    group's first facet weight) at x0 and at 0, where only the data term
//    remains;
//  * the solver initialised from x0 if F(x0) < F(0), else from zero.
#include <chrono>

#include "apikern.cuh"
#include "solver.cuh"

namespace fhs {

void unet_forward_device(fhs_unet* h, int n, int H, int W, const float* d_img, float* d_out);
int unet_device(const fhs_unet* h);

namespace {

template <class F>
fhs_status guarded_ws(F&& f) {
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
  } catch (...) {
    set_last_error("unknown error");
    return FHS_ERR_INVALID_ARG;
  }
}

// sum over channel c's visibilities (sorted order) of |Phi x - y|^2 per
// block: blocks of kMaxBlocksPerChannel accumulators in shared memory, one
// global atomic per CTA and block.  vis == nullptr: x = 0.
__global__ void block_residual_kernel(const float2* __restrict__ vis, const float2* __restrict__ y,
                                      const float4* __restrict__ geom, const int64_t* __restrict__ ch_voff,
                                      const int32_t* __restrict__ ch_M, const int32_t* __restrict__ ch_blkoff,
                                      double* __restrict__ out) {
  __shared__ double acc[kMaxBlocksPerChannel];
  const int c = blockIdx.y;
  if (threadIdx.x < kMaxBlocksPerChannel) acc[threadIdx.x] = 0.0;
  __syncthreads();
  const int64_t vo = ch_voff[c];
  const int M = ch_M[c];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    const float2 yv = y[vo + i];
    const float2 pv = vis ? vis[vo + i] : make_float2(0.f, 0.f);
    const double rx = (double)pv.x - yv.x, ry = (double)pv.y - yv.y;
    const int blk = (int)(__float_as_uint(geom[vo + i].z) >> 28);
    atomicAdd(&acc[blk], rx * rx + ry * ry);
  }
  __syncthreads();
  if (threadIdx.x < kMaxBlocksPerChannel && acc[threadIdx.x] != 0.0)
    atomicAdd(out + ch_blkoff[c] + threadIdx.x, acc[threadIdx.x]);
}

// sum_i sqrt(sum_l c_{l,i}^2) over the s coefficient rows of one group:
// rows below dirac_off from coef [lg][s], the Dirac rows from x / 3
__global__ void group_l21_kernel(const float* __restrict__ coef, const float* __restrict__ x, int64_t s,
                                 int64_t dirac_off, int64_t N, int lg, double* __restrict__ out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (int64_t)gridDim.x * blockDim.x) {
    double ss = 0.0;
    for (int l = 0; l < lg; ++l) {
      const double c = i < dirac_off ? (double)coef[(size_t)l * s + i]
                                     : (double)x[(size_t)l * N + (i - dirac_off)] * (1.0 / 3.0);
      ss += c * c;
    }
    acc += sqrt(ss);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

__global__ void clip0_kernel(float* __restrict__ x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = fmaxf(x[i], 0.f);
}

int grid_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

// data term sum_b max(0, ||y_b - Phi_b x|| - eps_b); x == nullptr: x = 0
double data_term(Solver* S, const float* x, float2* vis, DevBuf<double>& blk, cudaStream_t s) {
  MeasOp* op = S->op;
  if (x) measop_real_forward(op, x, vis, s);
  FHS_CUDA(cudaMemsetAsync(blk.p, 0, blk.n * sizeof(double), s));
  dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>((op->maxM + 255) / 256, 64)), op->L);
  block_residual_kernel<<<grid, 256, 0, s>>>(x ? vis : nullptr, S->y.p, op->geom.p, op->ch_voff.p, op->ch_M.p,
                                             op->ch_blkoff.p, blk.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  std::vector<double> h(op->nblk_tot);
  blk.download(h.data(), op->nblk_tot, s);
  FHS_CUDA(cudaStreamSynchronize(s));
  double f = 0.0;
  for (int b = 0; b < op->nblk_tot; ++b) f += std::max(0.0, std::sqrt(h[b]) - S->h_eps[b]);
  return f;
}

// sum_g gamma_g ||Psi^T x_g||_{2,1} + (nuclear priors) sum_g gamma0_g ||x_g||_*
double prior_terms(Solver* S, const float* x, cudaStream_t s) {
  const int G = S->G, lg = S->lg;
  const int64_t N = S->N;
  const SaraPlan& p = S->sp;
  DevBuf<float> coef, apx;
  coef.alloc((size_t)lg * p.s);
  apx.alloc((size_t)lg * p.apx_total);
  DevBuf<double> l21;
  l21.alloc(G);
  l21.zero(s);
  for (int g = 0; g < G; ++g) {
    const float* xg = x + (size_t)g * lg * N;
    sara_analysis(p, xg, coef.p, apx.p, lg, s);
    group_l21_kernel<<<grid_for(p.s), 256, 0, s>>>(coef.p, xg, p.s, p.boff[kSaraWavelets], N, lg, l21.p + g);
    count_launch();
    FHS_LAUNCH_CHECK();
  }
  std::vector<double> h_l21(G), h_nuc(G, 0.0);
  l21.download(h_l21.data(), G, s);
  if (S->nuclear) {
    // FP64 Gram of each whole sub-cube, as the standalone nuclear_norm
    DevBuf<double> xd, val;
    xd.alloc((size_t)S->L * N);
    val.alloc(G);
    launch_f2d(x, xd.p, (int64_t)S->L * N, s);
    NucPlan np;
    nuc_plan_init(np, (int)N, 1, 1, 1, {0, (int)N}, {0, 1}, 0, 0, FHS_WINDOW_NONE, 1, lg, s);
    for (int g = 0; g < G; ++g) {
      nuc_gram_fp64(np, xd.p + (size_t)g * lg * N, N, s);
      nuc_eig(np, nullptr, nullptr, val.p + g, s, 64.0 * lg * 2.220446049250313e-16);
    }
    val.download(h_nuc.data(), G, s);
  }
  FHS_CUDA(cudaStreamSynchronize(s));
  const int Q = (int)(S->gamma0.size() / std::max(G, 1));
  double f = 0.0;
  for (int g = 0; g < G; ++g) {
    f += S->gamma[g] * h_l21[g];
    if (S->nuclear && Q > 0) f += S->gamma0[(size_t)g * Q] * h_nuc[g];
  }
  return f;
}

}  // namespace
}  // namespace fhs

using namespace fhs;

extern "C" {

fhs_status fhs_solver_init_warm(fhs_solver* s_, fhs_unet* net, int chunk, fhs_warm_info* info) {
  return guarded_ws([&] {
    FHS_CHECK(s_ && net, FHS_ERR_INVALID_ARG, "null handle");
    Solver* S = reinterpret_cast<Solver*>(s_);
    FHS_CHECK(S->params_set && S->data_set, FHS_ERR_STATE, "set data and params before init");
    MeasOp* op = S->op;
    FHS_CHECK(!op->dr, FHS_ERR_UNSUPPORTED, "the warm start needs a visibility operator");
    FHS_CHECK(unet_device(net) == op->device, FHS_ERR_INVALID_ARG, "network and solver on different devices");
    FHS_CHECK(op->Ny % 8 == 0 && op->Nx % 8 == 0, FHS_ERR_UNSUPPORTED, "the network needs image sides divisible by 8");
    const auto t0 = std::chrono::steady_clock::now();
    DeviceGuard dg(op->device);
    cudaStream_t s = op->stream;
    const int L = S->L;
    const int64_t N = S->N, n = (int64_t)L * N;
    if (chunk <= 0) chunk = 16;
    DevBuf<float> dirty, psf, x0;
    DevBuf<float2> vis;
    DevBuf<double> peak, blk;
    dirty.alloc(n);
    psf.alloc(n);
    x0.alloc(n);
    vis.alloc(std::max<int64_t>(op->Mtot, 1));
    peak.alloc(L);
    blk.alloc(std::max(op->nblk_tot, 1));
    // dirty cube Re(Phi^H y), PSF peaks Re(Phi^H Phi delta) at the centre pixel
    measop_real_adjoint(op, S->y.p, dirty.p, s);
    FHS_CUDA(cudaMemsetAsync(psf.p, 0, (size_t)n * sizeof(float), s));
    launch_plane_set(psf.p, N, L, (int64_t)(op->Nx / 2) * op->Ny + op->Ny / 2, 1.f, s);
    measop_real_forward(op, psf.p, vis.p, s);
    measop_real_adjoint(op, vis.p, psf.p, s);
    launch_plane_max(psf.p, N, L, peak.p, s);
    launch_plane_scale_inv(dirty.p, N, L, peak.p, s);
    FHS_CUDA(cudaStreamSynchronize(s));
    // the network, chunk channels at a time ([Nx][Ny] images)
    for (int c0 = 0; c0 < L; c0 += chunk) {
      const int nc = std::min(chunk, L - c0);
      unet_forward_device(net, nc, op->Nx, op->Ny, dirty.p + (size_t)c0 * N, x0.p + (size_t)c0 * N);
    }
    clip0_kernel<<<grid_for(n), 256, 0, s>>>(x0.p, n);
    count_launch();
    FHS_LAUNCH_CHECK();
    // fallback rule
    const double f_cold = data_term(S, nullptr, vis.p, blk, s);
    const double f_warm = data_term(S, x0.p, vis.p, blk, s) + prior_terms(S, x0.p, s);
    const bool use = std::isfinite(f_warm) && f_warm < f_cold;
    solver_init_state(S, nullptr, use ? x0.p : nullptr);
    if (info) {
      info->used = use ? 1 : 0;
      info->objective_warm = f_warm;
      info->objective_cold = f_cold;
      info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
  });
}

}  // extern "C"
