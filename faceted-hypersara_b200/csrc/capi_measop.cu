// C-ABI entry points: library info and the measurement operator.
#include <cmath>
#include <random>

#include "apikern.cuh"
#include "measop.cuh"

namespace fhs {

static thread_local std::string t_last_error;
void set_last_error(const std::string& m) { t_last_error = m; }

// Runs f, translating exceptions into a status (no exception crosses the ABI).
template <class F>
static fhs_status guarded(F&& f) {
  try {
    f();
    t_last_error.clear();
    return FHS_OK;
  } catch (const Error& e) {
    t_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    t_last_error = "host allocation failed";
    return FHS_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    t_last_error = e.what();
    return FHS_ERR_INVALID_ARG;
  } catch (...) {
    t_last_error = "unknown error";
    return FHS_ERR_INVALID_ARG;
  }
}

static MeasOp* checked(fhs_measop* op) {
  FHS_CHECK(op != nullptr, FHS_ERR_INVALID_ARG, "null operator handle");
  return reinterpret_cast<MeasOp*>(op);
}
static MeasOp* committed(fhs_measop* op) {
  MeasOp* m = checked(op);
  FHS_CHECK(m->committed, FHS_ERR_STATE, "operator not committed (call fhs_measop_commit)");
  return m;
}

// Grows a device staging buffer of doubles.
static double* stage(MeasOp* op, size_t n) {
  if (op->stage.n < n) op->stage.alloc(n);
  return op->stage.p;
}
static float2* vis_scratch(MeasOp* op, DevBuf<float2>& b) {
  if (b.n < (size_t)std::max<int64_t>(op->Mtot, 1)) b.alloc(std::max<int64_t>(op->Mtot, 1));
  return b.p;
}
static float* img_scratch(MeasOp* op) {
  const size_t n = (size_t)op->L * op->Npix();
  if (op->img_a.n < n) op->img_a.alloc(n);
  return op->img_a.p;
}

void measop_real_forward(const MeasOp* op, const float* img, float2* vis, cudaStream_t s) {
  if (op->tw_y.p) {   // hand-written real-to-half-spectrum transforms
    fft_forward_half(op, img, 0, op->L, s);
    launch_degrid_plain(op, 0, op->L, vis, s, true);
  } else {
    launch_pad(op, img, 0, op->L, s);
    fft_forward(op, 0, op->L, s);
    launch_degrid_plain(op, 0, op->L, vis, s);
  }
}

void measop_real_adjoint(const MeasOp* op, const float2* vis, float* img, cudaStream_t s) {
  launch_grid_plain(op, 0, op->L, vis, s);
  if (op->tw_y.p) {   // hand-written spectrum-to-real transforms
    fft_inverse_real(op, img, 0, op->L, s);
    launch_scale_image(op, img, op->L, s);
  } else {
    fft_inverse(op, 0, op->L, s);
    launch_crop_real(op, img, nullptr, 0, op->L, s);
  }
}

// HS_forward_operator_G.m:36-52 (precond: HS_forward_operator_precond_G.m:40-55,
// y = sqrt(pU) .* G A x), all channels, host buffers.
static void forward_impl(MeasOp* op, const double* x, double* y, bool precond) {
  FHS_CHECK(x && y, FHS_ERR_INVALID_ARG, "null buffer");
  FHS_CHECK(!precond || op->precond, FHS_ERR_STATE, "no preconditioner set");
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  const int64_t N = op->Npix();
  double* st = stage(op, std::max<int64_t>(N * op->L, 2 * op->Mtot));
  float* img = img_scratch(op);
  float2* va = vis_scratch(op, op->vis_a);
  FHS_CUDA(cudaMemcpyAsync(st, x, N * op->L * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_d2f(st, img, N * op->L, s);
  measop_real_forward(op, img, va, s);
  if (precond) launch_scale_pu(op, va, true, s);
  launch_vis_scatter(va, st, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, op->L, op->maxM, 0, s);
  FHS_CUDA(cudaMemcpyAsync(y, st, 2 * op->Mtot * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
}

// HS_adjoint_operator_G.m:42-57 then real() (precond:
// HS_adjoint_operator_precond_G.m, x = At(G' (sqrt(pU) .* y))).
static void adjoint_impl(MeasOp* op, const double* y, double* x, bool precond) {
  FHS_CHECK(x && y, FHS_ERR_INVALID_ARG, "null buffer");
  FHS_CHECK(!precond || op->precond, FHS_ERR_STATE, "no preconditioner set");
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  const int64_t N = op->Npix();
  double* st = stage(op, std::max<int64_t>(N * op->L, 2 * op->Mtot));
  float* img = img_scratch(op);
  float2* va = vis_scratch(op, op->vis_a);
  FHS_CUDA(cudaMemcpyAsync(st, y, 2 * op->Mtot * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_vis_gather(st, va, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, op->L, op->maxM, 0, s);
  if (precond) launch_scale_pu(op, va, true, s);
  measop_real_adjoint(op, va, img, s);
  launch_f2d(img, st, N * op->L, s);
  FHS_CUDA(cudaMemcpyAsync(x, st, N * op->L * sizeof(double), cudaMemcpyDeviceToHost, s));
  FHS_CUDA(cudaStreamSynchronize(s));
}

// util_operator_norm.m:43-61: power iteration on Phi_l^H Phi_l per channel,
// Phi_l = G_l A (precond: sqrt(pU) G_l A, so the middle factor is pU).
static void operator_norm_impl(MeasOp* op, int max_iter, double tol, double* sq, bool precond) {
  FHS_CHECK(sq != nullptr && max_iter > 0, FHS_ERR_INVALID_ARG, "bad arguments");
  FHS_CHECK(!precond || op->precond, FHS_ERR_STATE, "no preconditioner set");
  DeviceGuard g(op->device);
  cudaStream_t s = op->stream;
  const int64_t N = op->Npix();
  const int L = op->L;
  float* img = img_scratch(op);
  float2* va = vis_scratch(op, op->vis_a);
  std::vector<float> h((size_t)N * L);
  std::mt19937_64 rng(12345);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (auto& v : h) v = nd(rng);
  FHS_CUDA(cudaMemcpyAsync(img, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, s));
  DevBuf<double> nrm;
  nrm.alloc(L);
  std::vector<double> hn(L), inv(L), val(L, 0.0);
  std::vector<char> done(L, 0);
  DevBuf<double> dinv;
  dinv.alloc(L);
  launch_plane_sumsq(img, N, L, nrm.p, s);
  nrm.download(hn.data(), L, s);
  FHS_CUDA(cudaStreamSynchronize(s));
  for (int l = 0; l < L; ++l) inv[l] = 1.0 / std::sqrt(hn[l]);
  dinv.upload(inv.data(), L, s);
  launch_plane_scale(img, N, L, dinv.p, s);
  for (int it = 0; it < max_iter; ++it) {
    launch_pad(op, img, 0, L, s);
    fft_forward(op, 0, L, s);
    launch_degrid_plain(op, 0, L, va, s);
    if (precond) launch_scale_pu(op, va, false, s);
    launch_grid_plain(op, 0, L, va, s);
    fft_inverse(op, 0, L, s);
    launch_crop_real(op, img, nullptr, 0, L, s);
    launch_plane_sumsq(img, N, L, nrm.p, s);
    nrm.download(hn.data(), L, s);
    FHS_CUDA(cudaStreamSynchronize(s));
    bool all = true;
    for (int l = 0; l < L; ++l) {
      const double nv = std::sqrt(hn[l]);
      FHS_CHECK(std::isfinite(nv), FHS_ERR_NUMERIC, "non-finite operator norm iterate");
      if (!done[l]) {
        if (std::fabs(nv - val[l]) <= tol * nv) done[l] = 1;
        val[l] = nv;
      }
      all = all && done[l];
      inv[l] = nv > 0 ? 1.0 / nv : 0.0;
    }
    if (all) break;
    dinv.upload(inv.data(), L, s);
    launch_plane_scale(img, N, L, dinv.p, s);
  }
  for (int l = 0; l < L; ++l) sq[l] = val[l];
}

}  // namespace fhs

using namespace fhs;

extern "C" {

int fhs_abi_version(void) { return FHS_ABI_VERSION; }
const char* fhs_last_error(void) { return t_last_error.c_str(); }
unsigned long long fhs_kernel_launch_count(void) { return g_launches; }

fhs_status fhs_measop_create(int device, int Ny, int Nx, int oy, int ox, int Jy, int Jx, int n_channels,
                             fhs_measop** out) {
  return guarded([&] {
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null output pointer");
    *out = reinterpret_cast<fhs_measop*>(measop_create(device, Ny, Nx, oy, ox, Jy, Jx, n_channels));
  });
}

fhs_status fhs_measop_destroy(fhs_measop* op) {
  return guarded([&] { delete reinterpret_cast<MeasOp*>(op); });
}

fhs_status fhs_measop_set_channel(fhs_measop* op, int channel, int64_t n_vis, const double* om_y,
                                  const double* om_x, const double* weights, int n_blocks,
                                  const int64_t* block_sizes) {
  return guarded([&] { measop_set_channel(checked(op), channel, n_vis, om_y, om_x, weights, n_blocks, block_sizes); });
}

fhs_status fhs_measop_commit(fhs_measop* op) {
  return guarded([&] { measop_commit(checked(op)); });
}

int64_t fhs_measop_n_vis(const fhs_measop* op, int channel) {
  const MeasOp* m = reinterpret_cast<const MeasOp*>(op);
  if (!m || channel < 0 || channel >= m->L) return -1;
  return m->ch[channel].M;
}

int fhs_measop_n_blocks(const fhs_measop* op, int channel) {
  const MeasOp* m = reinterpret_cast<const MeasOp*>(op);
  if (!m || channel < 0 || channel >= m->L) return -1;
  return (int)m->ch[channel].block_sizes.size();
}

fhs_status fhs_measop_image_size(const fhs_measop* op, int* Ny, int* Nx, int* n_channels) {
  return guarded([&] {
    const MeasOp* m = reinterpret_cast<const MeasOp*>(op);
    FHS_CHECK(m != nullptr, FHS_ERR_INVALID_ARG, "null operator");
    FHS_CHECK(Ny && Nx && n_channels, FHS_ERR_INVALID_ARG, "null output pointer");
    *Ny = m->Ny;
    *Nx = m->Nx;
    *n_channels = m->L;
  });
}

fhs_status fhs_measop_create_dr(fhs_measop* vis, fhs_measop** out) {
  return guarded([&] {
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    MeasOp* v = committed(vis);
    FHS_CHECK(!v->precond, FHS_ERR_UNSUPPORTED, "no dimensionality reduction of a preconditioned operator");
    *out = reinterpret_cast<fhs_measop*>(measop_create_dr(v));
  });
}

int fhs_measop_is_dr(const fhs_measop* op) {
  const MeasOp* m = reinterpret_cast<const MeasOp*>(op);
  return m ? (m->dr ? 1 : 0) : -1;
}

static MeasOp* dr_channel(fhs_measop* op_, int channel) {
  MeasOp* op = committed(op_);
  FHS_CHECK(op->dr, FHS_ERR_STATE, "not a dimensionality-reduced operator");
  FHS_CHECK(channel >= 0 && channel < op->L, FHS_ERR_INVALID_ARG, "bad channel index");
  return op;
}

fhs_status fhs_measop_dr_cells(fhs_measop* op_, int channel, int64_t* cells) {
  return guarded([&] {
    MeasOp* op = dr_channel(op_, channel);
    const int64_t n = op->h_M[channel];
    FHS_CHECK(n == 0 || cells, FHS_ERR_INVALID_ARG, "null buffer");
    if (n == 0) return;
    DeviceGuard g(op->device);
    std::vector<int32_t> h(n);
    op->dr_cell.download_at(h.data(), op->h_voff[channel], n, op->stream);
    FHS_CUDA(cudaStreamSynchronize(op->stream));
    for (int64_t i = 0; i < n; ++i) cells[i] = h[i];
  });
}

static void tuning_record(const MeasOp* op, fhs_tuning* t) {
  *t = fhs_tuning{};
  t->tuned = op->tuned ? 1 : 0;
  t->fft_chunk = op->own_fft || op->tw_y.p ? op->fft_chunk : -1;
  t->grid_slice = op->dr ? 0 : op->grid_slice;
  t->n_fft = (int)std::min<size_t>(op->tune_fft.size(), FHS_TUNING_MAX_CANDIDATES);
  for (int i = 0; i < t->n_fft; ++i) {
    t->fft_candidates[i] = op->tune_fft[i].first;
    t->fft_ms[i] = op->tune_fft[i].second;
  }
  t->n_grid = (int)std::min<size_t>(op->tune_grid.size(), FHS_TUNING_MAX_CANDIDATES);
  for (int i = 0; i < t->n_grid; ++i) {
    t->grid_candidates[i] = op->tune_grid[i].first;
    t->grid_ms[i] = op->tune_grid[i].second;
  }
}

fhs_status fhs_measop_autotune(fhs_measop* op_, fhs_tuning* out) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    measop_autotune(op);
    if (out) tuning_record(op, out);
  });
}

fhs_status fhs_measop_set_tuning(fhs_measop* op_, int fft_chunk, int grid_slice) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(fft_chunk >= 0 && grid_slice >= 1024, FHS_ERR_INVALID_ARG, "fft_chunk >= 0, grid_slice >= 1024");
    measop_set_grid_slice(op, grid_slice);
    op->fft_chunk = fft_chunk;
    op->tune_fft.clear();
    op->tune_grid.clear();
    op->tuned = true;
    ++op->layout_epoch;
  });
}

fhs_status fhs_measop_tuning(const fhs_measop* op_, fhs_tuning* out) {
  return guarded([&] {
    FHS_CHECK(out != nullptr, FHS_ERR_INVALID_ARG, "null output");
    tuning_record(committed(const_cast<fhs_measop*>(op_)), out);
  });
}

fhs_status fhs_measop_dr_lambda(fhs_measop* op_, int channel, double* lambda) {
  return guarded([&] {
    MeasOp* op = dr_channel(op_, channel);
    const int64_t n = op->h_M[channel];
    FHS_CHECK(n == 0 || lambda, FHS_ERR_INVALID_ARG, "null buffer");
    if (n == 0) return;
    DeviceGuard g(op->device);
    std::vector<int32_t> cell(n);
    op->dr_cell.download_at(cell.data(), op->h_voff[channel], n, op->stream);
    std::vector<float2> w((size_t)op->No());
    op->dr_omega.download_at(w.data(), (size_t)channel * op->No(), op->No(), op->stream);
    FHS_CUDA(cudaStreamSynchronize(op->stream));
    for (int64_t i = 0; i < n; ++i) lambda[i] = std::hypot((double)w[cell[i]].x, (double)w[cell[i]].y);
  });
}

int64_t fhs_measop_grid_size(const fhs_measop* op) {
  const MeasOp* m = reinterpret_cast<const MeasOp*>(op);
  return m ? m->No() : -1;
}

fhs_status fhs_scaled_fft(fhs_measop* op_, const double* x, double* Fx) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(x && Fx, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    const int64_t N = op->Npix(), No = op->No();
    double* st = stage(op, std::max<size_t>(N, 2 * No));
    float* img = img_scratch(op);
    FHS_CUDA(cudaMemcpyAsync(st, x, N * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_d2f(st, img, N, s);
    launch_pad(op, img, 0, 1, s);
    fft_forward(op, 0, 1, s);
    launch_grid_to_matlab(op->gridA.p, st, op->Ny, op->Nx, op->Ky, op->Kx, 1, s);
    FHS_CUDA(cudaMemcpyAsync(Fx, st, 2 * No * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_scaled_fft_adjoint(fhs_measop* op_, const double* Fx, double* xc) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(xc && Fx, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    const int64_t N = op->Npix(), No = op->No();
    double* st = stage(op, 2 * std::max<size_t>(N, No));
    FHS_CUDA(cudaMemcpyAsync(st, Fx, 2 * No * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_grid_from_matlab(st, op->gridB.p, op->Ny, op->Nx, op->Ky, op->Kx, 1, s);
    fft_inverse(op, 0, 1, s);
    launch_crop_complex(op->gridA.p, st, op->sy.p, op->sx.p, op->Ny, op->Nx, op->Ky, op->Kx, 1, s);
    // the gridding kernels never write empty tiles: restore the zeros of plane 0
    FHS_CUDA(cudaMemsetAsync(op->gridB.p, 0, No * sizeof(float2), s));
    FHS_CUDA(cudaMemcpyAsync(xc, st, 2 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_apply_direct_operator(fhs_measop* op_, int channel, const double* Fx, double* y) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(channel >= 0 && channel < op->L, FHS_ERR_INVALID_ARG, "bad channel");
    FHS_CHECK(Fx && y, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    const int64_t No = op->No(), M = op->h_M[channel];
    double* st = stage(op, 2 * std::max<int64_t>(No, M));
    float2* va = vis_scratch(op, op->vis_a);
    FHS_CUDA(cudaMemcpyAsync(st, Fx, 2 * No * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_grid_from_matlab(st, op->gridA.p + channel * No, op->Ny, op->Nx, op->Ky, op->Kx, 1, s);
    launch_degrid_plain(op, channel, 1, va, s);
    launch_vis_scatter(va, st, op->perm.p, op->ch_voff.p, op->ch_M.p, channel, 1, M, 0, s);
    FHS_CUDA(cudaMemcpyAsync(y, st, 2 * M * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_apply_adjoint_operator(fhs_measop* op_, int channel, const double* y, double* Fx) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(channel >= 0 && channel < op->L, FHS_ERR_INVALID_ARG, "bad channel");
    FHS_CHECK(Fx && y, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    const int64_t No = op->No(), M = op->h_M[channel];
    double* st = stage(op, 2 * std::max<int64_t>(No, M));
    float2* va = vis_scratch(op, op->vis_a);
    FHS_CUDA(cudaMemcpyAsync(st, y, 2 * M * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_vis_gather(st, va, op->perm.p, op->ch_voff.p, op->ch_M.p, channel, 1, M, 0, s);
    launch_grid_plain(op, channel, 1, va, s);
    launch_grid_to_matlab(op->gridB.p + channel * No, st, op->Ny, op->Nx, op->Ky, op->Kx, 1, s);
    FHS_CUDA(cudaMemcpyAsync(Fx, st, 2 * No * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_forward_operator(fhs_measop* op_, const double* x, double* y) {
  return guarded([&] { forward_impl(committed(op_), x, y, false); });
}

fhs_status fhs_adjoint_operator(fhs_measop* op_, const double* y, double* x) {
  return guarded([&] { adjoint_impl(committed(op_), y, x, false); });
}

fhs_status fhs_forward_operator_precond(fhs_measop* op_, const double* x, double* y) {
  return guarded([&] { forward_impl(committed(op_), x, y, true); });
}

fhs_status fhs_adjoint_operator_precond(fhs_measop* op_, const double* y, double* x) {
  return guarded([&] { adjoint_impl(committed(op_), y, x, true); });
}

fhs_status fhs_measop_set_preconditioner(fhs_measop* op_, int channel, const double* pU) {
  return guarded([&] { measop_set_preconditioner(committed(op_), channel, pU); });
}

fhs_status fhs_gen_preconditioning_matrix(int64_t n_vis, const double* om_y, const double* om_x, int Ky, int Kx,
                                          int sub_pixels, double* pU) {
  return guarded([&] { gen_uniform_weights(n_vis, om_y, om_x, Ky, Kx, sub_pixels, pU); });
}

fhs_status fhs_compute_residual_images(fhs_measop* op_, const double* y, const double* x, double* res) {
  return guarded([&] {
    MeasOp* op = committed(op_);
    FHS_CHECK(y && x && res, FHS_ERR_INVALID_ARG, "null buffer");
    DeviceGuard g(op->device);
    cudaStream_t s = op->stream;
    const int64_t N = op->Npix();
    const int L = op->L;
    double* st = stage(op, std::max<int64_t>(N * L, 2 * op->Mtot));
    float* img = img_scratch(op);
    float2* va = vis_scratch(op, op->vis_a);
    float2* vb = vis_scratch(op, op->vis_b);
    DevBuf<float> psf;
    psf.alloc((size_t)N * L);
    DevBuf<double> peak;
    peak.alloc(L);
    // residual visibilities y - G A x
    FHS_CUDA(cudaMemcpyAsync(st, y, 2 * op->Mtot * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_vis_gather(st, vb, op->perm.p, op->ch_voff.p, op->ch_M.p, 0, L, op->maxM, 0, s);
    FHS_CUDA(cudaMemcpyAsync(st, x, N * L * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_d2f(st, img, N * L, s);
    launch_pad(op, img, 0, L, s);
    fft_forward(op, 0, L, s);
    launch_degrid_plain(op, 0, L, va, s);
    launch_vis_axpy(vb, va, -1.f, op->Mtot, s);  // vb <- y - G A x
    launch_grid_plain(op, 0, L, vb, s);
    fft_inverse(op, 0, L, s);
    launch_crop_real(op, img, nullptr, 0, L, s);
    // PSF: a dirac at (N/2, N/2) (0-based) through G^H G A
    FHS_CUDA(cudaMemsetAsync(psf.p, 0, (size_t)N * L * sizeof(float), s));
    launch_plane_set(psf.p, N, L, (int64_t)(op->Nx / 2) * op->Ny + op->Ny / 2, 1.f, s);
    launch_pad(op, psf.p, 0, L, s);
    fft_forward(op, 0, L, s);
    launch_degrid_plain(op, 0, L, va, s);
    launch_grid_plain(op, 0, L, va, s);
    fft_inverse(op, 0, L, s);
    launch_crop_real(op, psf.p, nullptr, 0, L, s);
    launch_plane_max(psf.p, N, L, peak.p, s);
    launch_plane_scale_inv(img, N, L, peak.p, s);
    launch_f2d(img, st, N * L, s);
    FHS_CUDA(cudaMemcpyAsync(res, st, N * L * sizeof(double), cudaMemcpyDeviceToHost, s));
    FHS_CUDA(cudaStreamSynchronize(s));
  });
}

fhs_status fhs_operator_norm(fhs_measop* op_, int max_iter, double tol, double* sq) {
  return guarded([&] { operator_norm_impl(committed(op_), max_iter, tol, sq, false); });
}

fhs_status fhs_operator_norm_precond(fhs_measop* op_, int max_iter, double tol, double* sq) {
  return guarded([&] { operator_norm_impl(committed(op_), max_iter, tol, sq, true); });
}

}  // extern "C"
