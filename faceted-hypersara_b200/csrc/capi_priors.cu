// C-ABI entry points: standalone prior functions and the host-buffer data
// fidelity step (src/proj_l2ball.m, src/nuclear_norm.m, src/compute_sara_prior.m,
// SARA Psit / Psi, src/update_dual_data_fidelity.m).
#include <cmath>

#include "apikern.cuh"
#include "measop.cuh"
#include "nuclear.cuh"
#include "sara.cuh"

namespace fhs {

namespace {

template <class F>
fhs_status guarded_p(F&& f) {
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

// Device + stream for a standalone call.
struct Ctx {
  DeviceGuard g;
  cudaStream_t s = nullptr;
  explicit Ctx(int device) : g(check_device(device)) { FHS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~Ctx() {
    if (s) cudaStreamDestroy(s);
  }
  static int check_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(FHS_ERR_NO_DEVICE, "no CUDA device available");
    FHS_CHECK(device >= 0 && device < n, FHS_ERR_INVALID_ARG, "bad device index");
    return device;
  }
};

__global__ void diff_sumsq_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                  double* __restrict__ out) {
  __shared__ double sh[256];
  double a = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double d = x[i] - y[i];
    a += d * d;
  }
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

__global__ void proj_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                            const double* __restrict__ part, int nparts, double eps, double* __restrict__ p) {
  __shared__ double scale;
  if (threadIdx.x == 0) {
    double s2 = 0;
    for (int i = 0; i < nparts; ++i) s2 += part[i];
    const double nrm = sqrt(s2);
    scale = nrm > 0 ? fmin(eps / nrm, 1.0) : 1.0;
  }
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = y[i] + (x[i] - y[i]) * scale;
}

__global__ void sumsq_rows_kernel(const float* __restrict__ coef, const float* __restrict__ x, int64_t s,
                                  int64_t dirac_off, int64_t npix, int L, double* __restrict__ part) {
  __shared__ double sh[256];
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (int64_t)gridDim.x * blockDim.x) {
    double ss = 0;
    for (int l = 0; l < L; ++l) {
      const float c = i < dirac_off ? coef[(size_t)l * s + i] : x[(size_t)l * npix + (i - dirac_off)] * (1.f / 3.f);
      ss += (double)c * c;
    }
    acc += sqrt(ss);
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

int nb(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 8); }

}  // namespace
}  // namespace fhs

using namespace fhs;

extern "C" {

fhs_status fhs_proj_l2ball(int device, int64_t n, const double* x, double eps, const double* y, double* p) {
  return guarded_p([&] {
    FHS_CHECK(n >= 0 && x && y && p, FHS_ERR_INVALID_ARG, "bad arguments");
    FHS_CHECK(std::isfinite(eps) && eps >= 0, FHS_ERR_INVALID_ARG, "eps must be finite and >= 0");
    if (n == 0) return;
    Ctx c(device);
    const int64_t m = 2 * n;  // complex as interleaved doubles
    DevBuf<double> dx, dy, dp, part;
    dx.alloc(m);
    dy.alloc(m);
    dp.alloc(m);
    const int blocks = nb(m);
    part.alloc(blocks);
    dx.upload(x, m, c.s);
    dy.upload(y, m, c.s);
    diff_sumsq_kernel<<<blocks, 256, 0, c.s>>>(dx.p, dy.p, m, part.p);
    count_launch();
    FHS_LAUNCH_CHECK();
    proj_kernel<<<blocks, 256, 0, c.s>>>(dx.p, dy.p, m, part.p, blocks, eps, dp.p);
    count_launch();
    FHS_LAUNCH_CHECK();
    dp.download(p, m, c.s);
    FHS_CUDA(cudaStreamSynchronize(c.s));
  });
}

fhs_status fhs_nuclear_norm(int device, int64_t n_pixels, int L, const double* x, double* f) {
  return guarded_p([&] {
    FHS_CHECK(n_pixels > 0 && n_pixels < (1LL << 31) && L >= 1 && x && f, FHS_ERR_INVALID_ARG, "bad arguments");
    FHS_CHECK(L <= kNucMaxL, FHS_ERR_UNSUPPORTED, "nuclear_norm supports at most 64 channels");
    Ctx c(device);
    const int64_t n = n_pixels * L;
    DevBuf<double> st;
    st.alloc(n);
    st.upload(x, n, c.s);
    NucPlan p;
    nuc_plan_init(p, (int)n_pixels, 1, 1, 1, {0, (int)n_pixels}, {0, 1}, 0, 0, FHS_WINDOW_NONE, 1, L, c.s);
    DevBuf<double> val;
    val.alloc(1);
    // FP64 Gram: the small singular values of a nearly low-rank cube need it
    // (svd() of the reference is FP64)
    nuc_gram_fp64(p, st.p, n_pixels, c.s);
    nuc_eig(p, nullptr, nullptr, val.p, c.s, 64.0 * L * 2.220446049250313e-16);
    val.download(f, 1, c.s);
    FHS_CUDA(cudaStreamSynchronize(c.s));
  });
}

int64_t fhs_sara_n_coefs(int Ny, int Nx, int nlevel) {
  try {
    return sara_plan(Ny, Nx, nlevel).s;
  } catch (...) {
    return -1;
  }
}

fhs_status fhs_sara_analysis(int device, int Ny, int Nx, int L, int nlevel, const double* x, double* coefs) {
  return guarded_p([&] {
    FHS_CHECK(L >= 1 && x && coefs, FHS_ERR_INVALID_ARG, "bad arguments");
    const SaraPlan p = sara_plan(Ny, Nx, nlevel);
    Ctx c(device);
    const int64_t N = (int64_t)Ny * Nx;
    DevBuf<double> st;
    st.alloc(std::max<int64_t>(N, p.s) * L);
    DevBuf<float> xf, cf, apx;
    xf.alloc(N * L);
    cf.alloc(p.s * L);
    apx.alloc(p.apx_total * L);
    st.upload(x, N * L, c.s);
    launch_d2f(st.p, xf.p, N * L, c.s);
    sara_analysis(p, xf.p, cf.p, apx.p, L, c.s);
    sara_dirac(p, xf.p, cf.p, L, c.s);
    launch_f2d(cf.p, st.p, p.s * L, c.s);
    st.download(coefs, p.s * L, c.s);
    FHS_CUDA(cudaStreamSynchronize(c.s));
  });
}

fhs_status fhs_sara_synthesis(int device, int Ny, int Nx, int L, int nlevel, const double* coefs, double* x) {
  return guarded_p([&] {
    FHS_CHECK(L >= 1 && x && coefs, FHS_ERR_INVALID_ARG, "bad arguments");
    const SaraPlan p = sara_plan(Ny, Nx, nlevel);
    Ctx c(device);
    const int64_t N = (int64_t)Ny * Nx;
    DevBuf<double> st;
    st.alloc(std::max<int64_t>(N, p.s) * L);
    DevBuf<float> xf, cf, apx;
    xf.alloc(N * L);
    cf.alloc(p.s * L);
    apx.alloc(p.apx_total * L);
    st.upload(coefs, p.s * L, c.s);
    launch_d2f(st.p, cf.p, p.s * L, c.s);
    sara_synthesis(p, cf.p, xf.p, apx.p, L, 1.f, c.s);
    launch_f2d(xf.p, st.p, N * L, c.s);
    st.download(x, N * L, c.s);
    FHS_CUDA(cudaStreamSynchronize(c.s));
  });
}

fhs_status fhs_compute_sara_prior(int device, int Ny, int Nx, int L, int nlevel, const double* x, double* f) {
  return guarded_p([&] {
    FHS_CHECK(L >= 1 && x && f, FHS_ERR_INVALID_ARG, "bad arguments");
    const SaraPlan p = sara_plan(Ny, Nx, nlevel);
    Ctx c(device);
    const int64_t N = (int64_t)Ny * Nx;
    DevBuf<double> st, part;
    st.alloc(N * L);
    DevBuf<float> xf, cf, apx;
    xf.alloc(N * L);
    cf.alloc(p.s * L);
    apx.alloc(p.apx_total * L);
    st.upload(x, N * L, c.s);
    launch_d2f(st.p, xf.p, N * L, c.s);
    sara_analysis(p, xf.p, cf.p, apx.p, L, c.s);
    const int blocks = nb(p.s);
    part.alloc(blocks);
    sumsq_rows_kernel<<<blocks, 256, 0, c.s>>>(cf.p, xf.p, p.s, p.boff[kSaraWavelets], N, L, part.p);
    count_launch();
    FHS_LAUNCH_CHECK();
    std::vector<double> h(blocks);
    part.download(h.data(), blocks, c.s);
    FHS_CUDA(cudaStreamSynchronize(c.s));
    double tot = 0;
    for (double v : h) tot += v;
    *f = tot;
  });
}

// update_dual_data_fidelity on host buffers: the solver's fused passes with
// G Fx_old taken from the caller's Fx_old grid (linearity of G).
}  // extern "C"

namespace fhs {
namespace {

// src/update_dual_data_fidelity.m:116-147 (no DR) on host buffers: the
// l2-ball form (pU = 1, :83) or, with precond, the ellipsoid projection
// (:126-147) warm-started from proj.
void dual_impl(MeasOp* op, double* v2, double* proj, const double* y, const double* x, double* Fx_old,
               const double* epsilon, const double* sigma22, double* Ftx, double* norm_res,
               double* global_norm_res, double* norm_epsilon, bool precond, int max_itr, int min_itr,
               double stop, int* fb_iters) {
  FHS_CHECK(v2 && y && x && Fx_old && epsilon && sigma22 && Ftx && norm_res, FHS_ERR_INVALID_ARG,
            "null argument");
  FHS_CHECK(op->committed, FHS_ERR_STATE, "operator not committed");
  if (precond) {
    FHS_CHECK(proj != nullptr, FHS_ERR_INVALID_ARG, "null proj");
    FHS_CHECK(op->precond, FHS_ERR_STATE, "no preconditioner set (fhs_measop_set_preconditioner)");
    FHS_CHECK(max_itr >= 1 && min_itr >= 0 && stop >= 0, FHS_ERR_INVALID_ARG, "bad ellipsoid-projection parameters");
  }
  DeviceGuard dg(op->device);
  cudaStream_t s = op->stream;
  const int L = op->L;
  const int64_t N = op->Npix(), No = op->No(), M = op->Mtot;
  const int64_t stage_n = std::max<int64_t>(std::max<int64_t>(2 * No * L, 2 * M), N * L);
  if (op->stage.n < (size_t)stage_n) op->stage.alloc(stage_n);
  if (op->vis_a.n < (size_t)std::max<int64_t>(M, 1)) op->vis_a.alloc(std::max<int64_t>(M, 1));
  if (op->vis_b.n < (size_t)std::max<int64_t>(M, 1)) op->vis_b.alloc(std::max<int64_t>(M, 1));
  DevBuf<float2> yd;
  yd.alloc(std::max<int64_t>(M, 1));
  DevBuf<double2> wd;
  if (precond) wd.alloc(std::max<int64_t>(M, 1));
  DevBuf<float> img, s22;
  img.alloc(N * L);
  s22.alloc(L);
  std::vector<float> hs(sigma22, sigma22 + L);
  s22.upload(hs.data(), L, s);
  double* st = op->stage.p;
  // G Fx_old -> vis_b (gold)
  FHS_CUDA(cudaMemcpyAsync(st, Fx_old, 2 * No * L * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_grid_from_matlab(st, op->gridA.p, op->Ny, op->Nx, op->Ky, op->Kx, L, s);
  launch_degrid_plain(op, 0, L, op->vis_b.p, s);
  // y, v2 -> sorted
  FHS_CUDA(cudaMemcpyAsync(st, y, 2 * M * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_vis_gather(st, yd.p, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, L, op->maxM, 0, s);
  FHS_CUDA(cudaMemcpyAsync(st, v2, 2 * M * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_vis_gather(st, op->vis_a.p, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, L, op->maxM, 0, s);
  if (precond) {  // w = proj - y (FP64)
    FHS_CUDA(cudaMemcpyAsync(st, proj, 2 * M * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_w_from_proj(op, st, yd.p, wd.p, s);
  }
  std::vector<double> e((size_t)L * kMaxBlocksPerChannel, 0.0);
  double eps2 = 0;
  for (int l = 0; l < L; ++l)
    for (int b = 0; b < op->h_nblk[l]; ++b) {
      const double v = epsilon[op->h_blkoff[l] + b];
      e[(size_t)l * kMaxBlocksPerChannel + b] = v;
      eps2 += v * v;
    }
  op->blk_eps.upload(e.data(), e.size(), s);
  // A x
  FHS_CUDA(cudaMemcpyAsync(st, x, N * L * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_d2f(st, img.p, N * L, s);
  launch_pad(op, img.p, 0, L, s);
  fft_forward(op, 0, L, s);
  launch_grid_to_matlab(op->gridA.p, st, op->Ny, op->Nx, op->Ky, op->Kx, L, s);
  FHS_CUDA(cudaMemcpyAsync(Fx_old, st, 2 * No * L * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
  // fused passes
  if (precond) {
    launch_degrid_dual_precond(op, 0, L, op->vis_a.p, op->vis_b.p, yd.p, wd.p, s);
    launch_block_reduce_precond(op, 0, L, s);
    launch_fb_iterations(op, 0, L, wd.p, yd.p, max_itr, min_itr, stop, s);
    launch_grid_dual_precond(op, 0, L, op->vis_a.p, wd.p, s);
  } else {
    launch_degrid_dual(op, 0, L, op->vis_a.p, op->vis_b.p, yd.p, s);
    launch_block_reduce(op, 0, L, s);
    launch_grid_dual(op, 0, L, op->vis_a.p, s);
  }
  fft_inverse(op, 0, L, s);
  launch_crop_real(op, img.p, s22.p, 0, L, s);
  launch_f2d(img.p, st, N * L, s);
  FHS_CUDA(cudaMemcpyAsync(Ftx, st, N * L * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
  launch_vis_scatter(op->vis_a.p, st, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, L, op->maxM, 0, s);
  FHS_CUDA(cudaMemcpyAsync(v2, st, 2 * M * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
  if (precond) {
    launch_proj_from_w(op, wd.p, yd.p, st, s);
    FHS_CUDA(cudaMemcpyAsync(proj, st, 2 * M * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  std::vector<double> stats((size_t)op->nblk_tot * 2);
  op->blk_stats.download(stats.data(), stats.size(), s);
  std::vector<int> cnt;
  if (precond && fb_iters) {
    cnt.resize((size_t)L * kMaxBlocksPerChannel);
    op->fb_count.download(cnt.data(), cnt.size(), s);
  }
  FHS_CUDA(cudaStreamSynchronize(s));
  double gres = 0;
  for (int b = 0; b < op->nblk_tot; ++b) {
    norm_res[b] = std::sqrt(stats[2 * b + 1]);
    gres += stats[2 * b + 1];
  }
  if (precond && fb_iters)
    for (int l = 0; l < L; ++l)
      for (int b = 0; b < op->h_nblk[l]; ++b) fb_iters[op->h_blkoff[l] + b] = cnt[(size_t)l * kMaxBlocksPerChannel + b];
  if (global_norm_res) *global_norm_res = gres;
  if (norm_epsilon) *norm_epsilon = eps2;
}

}  // namespace
}  // namespace fhs

extern "C" {

fhs_status fhs_update_dual_data_fidelity(fhs_measop* op_, double* v2, const double* y, const double* x,
                                         double* Fx_old, const double* epsilon, const double* sigma22,
                                         double* Ftx, double* norm_res, double* global_norm_res,
                                         double* norm_epsilon) {
  return guarded_p([&] {
    FHS_CHECK(op_ != nullptr, FHS_ERR_INVALID_ARG, "null operator handle");
    dual_impl(reinterpret_cast<MeasOp*>(op_), v2, nullptr, y, x, Fx_old, epsilon, sigma22, Ftx, norm_res,
              global_norm_res, norm_epsilon, false, 0, 0, 0.0, nullptr);
  });
}

fhs_status fhs_update_dual_data_fidelity_precond(fhs_measop* op_, double* v2, double* proj, const double* y,
                                                 const double* x, double* Fx_old, const double* epsilon,
                                                 int elipse_proj_max_iter, int elipse_proj_min_iter,
                                                 double elipse_proj_eps, const double* sigma22, double* Ftx,
                                                 double* norm_res, double* global_norm_res,
                                                 double* norm_epsilon, int* fb_iters) {
  return guarded_p([&] {
    FHS_CHECK(op_ != nullptr, FHS_ERR_INVALID_ARG, "null operator handle");
    dual_impl(reinterpret_cast<MeasOp*>(op_), v2, proj, y, x, Fx_old, epsilon, sigma22, Ftx, norm_res,
              global_norm_res, norm_epsilon, true, elipse_proj_max_iter, elipse_proj_min_iter, elipse_proj_eps,
              fb_iters);
  });
}

}  // extern "C"
