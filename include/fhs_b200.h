/*
 * fhs_b200.h -- C ABI of the B200 (sm_100a) Faceted HyperSARA library.
 *
 * Drop-in boundary for the reference's MATLAB entry points
 * (basp-group/Faceted-HyperSARA).  A MEX gateway (or ctypes, or a C program)
 * binds these functions; every buffer is a plain host pointer in MATLAB's
 * memory order:
 *   - image cubes  x[Ny, Nx, L]  double, column-major (y fastest);
 *   - grids        Fx[No]        complex double, interleaved (re, im),
 *                  column-major over (Ky = oy*Ny, Kx = ox*Nx);
 *   - visibilities y[M]          complex double, interleaved, channel after
 *                  channel, blocks of a channel concatenated in block order.
 * The library copies host buffers in and out and owns all device memory of a
 * handle.  No exception, exit() or abort() crosses this boundary: every call
 * returns an fhs_status and fhs_last_error() gives the message (thread-local).
 * A handle binds one CUDA device and one stream; handles are independent and
 * may be used from different host threads, one thread per handle at a time.
 */
#ifndef FHS_B200_H
#define FHS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FHS_ABI_VERSION 1

#if defined(__GNUC__)
#define FHS_API __attribute__((visibility("default")))
#else
#define FHS_API
#endif

typedef enum fhs_status {
  FHS_OK = 0,
  FHS_ERR_INVALID_ARG = 1,   /* bad size, index, pointer or parameter */
  FHS_ERR_CUDA = 2,          /* CUDA runtime / cuFFT failure */
  FHS_ERR_OUT_OF_MEMORY = 3, /* device allocation failed */
  FHS_ERR_STATE = 4,         /* call made in the wrong order */
  FHS_ERR_NUMERIC = 5,       /* non-finite value detected */
  FHS_ERR_UNSUPPORTED = 6,   /* configuration outside the supported limits */
  FHS_ERR_NO_DEVICE = 7      /* no CUDA device / driver */
} fhs_status;

/* ABI version of the loaded library (FHS_ABI_VERSION it was built with). */
FHS_API int fhs_abi_version(void);
/* Message of the last failed call on this host thread ("" if none). */
FHS_API const char* fhs_last_error(void);
/* Number of kernels this library launched since load (all handles). */
FHS_API unsigned long long fhs_kernel_launch_count(void);

/* ======================================================================
 * Measurement operator  Phi_l = G_l A  (replaces op_p_nufft of the
 * RI-measurement-operator submodule, built at
 * lib/operators/util_gen_measurement_operator_synth.m:86 and applied by
 * lib/operators/HS_forward_operator_G.m:36-52 / HS_adjoint_operator_G.m:42-57).
 * Min-max interpolation (Fessler & Sutton 2003), J taps per axis, 2-D
 * separable, scaling factors from a Kaiser-Bessel cosine series.
 * Limits: Ky = oy*Ny and Kx = ox*Nx multiples of 8 and <= 16384, Ny and Nx
 * even, 2 <= J <= 8, at most 16 blocks per channel.  The mask W of the
 * reference is the full grid (every G column is addressable).
 * ====================================================================== */
typedef struct fhs_measop fhs_measop;

FHS_API fhs_status fhs_measop_create(int device, int Ny, int Nx, int oy, int ox, int Jy, int Jx,
                             int n_channels, fhs_measop** out);
FHS_API fhs_status fhs_measop_destroy(fhs_measop* op);
/* Visibilities of one channel: frequencies (radians, om_y = v, om_x = u as
 * in op_p_nufft([{v} {u}], ...)), optional per-visibility weights (the noise
 * whitening folded into G's rows; NULL = 1), block sizes summing to n_vis. */
FHS_API fhs_status fhs_measop_set_channel(fhs_measop* op, int channel, int64_t n_vis, const double* om_y,
                                  const double* om_x, const double* weights, int n_blocks,
                                  const int64_t* block_sizes);
/* Finalise (device upload, visibility binning, FFT plans).  Required once
 * after all channels are set and before any apply call. */
FHS_API fhs_status fhs_measop_commit(fhs_measop* op);
FHS_API int64_t fhs_measop_n_vis(const fhs_measop* op, int channel);
FHS_API int64_t fhs_measop_grid_size(const fhs_measop* op); /* No = Ky*Kx */
/* Blocks of a channel as set by fhs_measop_set_channel (-1: bad channel);
 * the cell {l}{b} count of y / epsilon in update_dual_data_fidelity.m:1-6. */
FHS_API int fhs_measop_n_blocks(const fhs_measop* op, int channel);
/* Image size [Ny, Nx] and channel count L of x in the calls below (the
 * [M, N, L] of facetHyperSARA.m:1-6); host-side, needs no device. */
FHS_API fhs_status fhs_measop_image_size(const fhs_measop* op, int* Ny, int* Nx, int* n_channels);

/* A (op_nufft's scaled zero-padded FFT; shape contract of
 * src/apply_scaled_fourier_transform.m:21-24): x[Ny,Nx] -> Fx[No] complex. */
FHS_API fhs_status fhs_scaled_fft(fhs_measop* op, const double* x, double* Fx);
/* At (exact adjoint of A): Fx[No] complex -> x[Ny,Nx] complex. */
FHS_API fhs_status fhs_scaled_fft_adjoint(fhs_measop* op, const double* Fx, double* x_complex);
/* src/apply_direct_operator.m:1  y = G Fx  (Lambda = 1, no DR). */
FHS_API fhs_status fhs_apply_direct_operator(fhs_measop* op, int channel, const double* Fx, double* y);
/* src/apply_adjoint_operator.m:1  Fx = G' y  (Lambda = 1, no DR). */
FHS_API fhs_status fhs_apply_adjoint_operator(fhs_measop* op, int channel, const double* y, double* Fx);
/* lib/operators/HS_forward_operator_G.m:36-52: x[Ny,Nx,L] -> y (all channels). */
FHS_API fhs_status fhs_forward_operator(fhs_measop* op, const double* x, double* y);
/* lib/operators/HS_adjoint_operator_G.m:42-57 followed by real(): y -> x[Ny,Nx,L]. */
FHS_API fhs_status fhs_adjoint_operator(fhs_measop* op, const double* y, double* x);
/* src/compute_residual_images.m:83-102 (no DR): res[Ny,Nx,L] =
 * real(At(G'(y - G A x))) per channel, divided by the peak of the PSF
 * real(At(G'G A dirac)) with the dirac at pixel (Ny/2+1, Nx/2+1) (1-based). */
FHS_API fhs_status fhs_compute_residual_images(fhs_measop* op, const double* y, const double* x, double* res);
/* lib/utils/util_operator_norm.m:43-61: per-channel ||G_l A||^2 by power
 * iteration (op_norm of the submodule), FP32 operators, FP64 norms. */
FHS_API fhs_status fhs_operator_norm(fhs_measop* op, int max_iter, double tol, double* squared_norms);

/* src/update_dual_data_fidelity.m:116-147 (pU = 1, no DR) on host buffers.
 * v2, y: all channels' visibilities; x[Ny,Nx,L]; Fx_old[No,L] complex
 * (updated to A(x)); epsilon: one per block (channel-major); sigma22[L].
 * Outputs: v2 (updated), Ftx[Ny,Nx,L], norm_res (one per block),
 * global_norm_res and norm_epsilon (sums of squares, as the reference). */
FHS_API fhs_status fhs_update_dual_data_fidelity(fhs_measop* op, double* v2, const double* y,
                                         const double* x, double* Fx_old, const double* epsilon,
                                         const double* sigma22, double* Ftx, double* norm_res,
                                         double* global_norm_res, double* norm_epsilon);

/* ----------------------------------------------------------------------
 * Preconditioning and the ellipsoid projection (default non-DR data term of
 * the reference: src/update_dual_data_fidelity.m:126-147,
 * src/sara/sara.m:561-562,594-595)
 * ---------------------------------------------------------------------- */
/* util_gen_preconditioning_matrix (RI-measurement-operator submodule, set up
 * at imaging/imaging.m:436-438) with gen_uniform_weight_matrix = true:
 * pU[m] = 1 / (number of visibilities in the cell of visibility m on a
 * (Ky sub_pixels) x (Kx sub_pixels) grid, cells centred on the grid points).
 * Host computation over n_vis frequencies (radians). */
FHS_API fhs_status fhs_gen_preconditioning_matrix(int64_t n_vis, const double* om_y, const double* om_x, int Ky,
                                                  int Kx, int sub_pixels, double* pU);
/* Attaches the diagonal preconditioner aW{l} of one channel (all blocks, in
 * the channel's visibility order; entries finite and > 0).  Needs a committed
 * operator.  Once every channel has one, the *_precond calls below work and a
 * solver initialised afterwards runs the ellipsoid projection. */
FHS_API fhs_status fhs_measop_set_preconditioner(fhs_measop* op, int channel, const double* pU);
/* lib/operators/HS_forward_operator_precond_G.m:40-55: y = sqrt(pU) .* G A x. */
FHS_API fhs_status fhs_forward_operator_precond(fhs_measop* op, const double* x, double* y);
/* lib/operators/HS_adjoint_operator_precond_G.m: x = real(At(G' (sqrt(pU) .* y))). */
FHS_API fhs_status fhs_adjoint_operator_precond(fhs_measop* op, const double* y, double* x);
/* lib/utils/util_operator_norm.m:46-52: per-channel ||sqrt(pU) G_l A||^2
 * (squared_operator_norm_precond, the nu2 of imaging/imaging.m:846). */
FHS_API fhs_status fhs_operator_norm_precond(fhs_measop* op, int max_iter, double tol, double* squared_norms);
/* src/update_dual_data_fidelity.m:126-147 (no DR) on host buffers:
 * proj = solver_proj_elipse_fb(v2 ./ pU, r2, y, pU, eps, proj, max, min, eps_stop),
 * v2 = v2 + pU .* (r2 - proj), forward-backward iterations with step
 * mu = min(pU) per block, stopped when ||proj_k - proj_{k-1}|| <= eps_stop
 * ||proj_k|| after at least min iterations or at max iterations.  Arguments
 * as fhs_update_dual_data_fidelity plus proj (in/out, all visibilities) and
 * fb_iters (optional out, FB iterations run per block). */
FHS_API fhs_status fhs_update_dual_data_fidelity_precond(fhs_measop* op, double* v2, double* proj,
                                                         const double* y, const double* x, double* Fx_old,
                                                         const double* epsilon, int elipse_proj_max_iter,
                                                         int elipse_proj_min_iter, double elipse_proj_eps,
                                                         const double* sigma22, double* Ftx, double* norm_res,
                                                         double* global_norm_res, double* norm_epsilon,
                                                         int* fb_iters);

/* ----------------------------------------------------------------------
 * Visibility gridding / dimensionality reduction (DR): the operator built by
 * lib/operators/util_load_data_gen_dr_measurement_operator.m:109-228 and the
 * flag_visibility_gridding branches of update_dual_data_fidelity.m:85-125,
 * HS_forward_operator_G.m:41-45, HS_adjoint_operator_G.m:46-49,
 * compute_residual_images.m:42-80 and util_operator_norm.m
 * ---------------------------------------------------------------------- */
/* Builds the DR operator of a committed visibility operator: per channel
 * H = G'G over all its blocks, W = diag(H) > 0, Lambda = diag(H)^-1/2 on W,
 * one data block per channel (the reference's "1 single block per channel").
 * The result is a committed operator of the same image and grid sizes whose
 * data entries of channel l are the n_vis(l) = |W_l| active grid cells in
 * column-major order (the order of MATLAB's Fx(W)).  On it the calls above
 * apply the reference's DR formulas: apply_direct / forward: y =
 * Lambda .* (H Fx)(W); apply_adjoint / adjoint: g2(W) = H (Lambda .* y);
 * residual images, operator norm, the l2-ball dual update and the solvers
 * likewise.  No preconditioner (util_load_data_gen_dr_measurement_operator.m:
 * 118).  The visibility operator stays valid and independent. */
FHS_API fhs_status fhs_measop_create_dr(fhs_measop* vis_op, fhs_measop** dr_op);
/* 1 for an operator made by fhs_measop_create_dr, 0 otherwise, -1 null. */
FHS_API int fhs_measop_is_dr(const fhs_measop* op);
/* W{l}: the 0-based column-major grid index of each data entry of channel l
 * (n_vis(l) values). */
FHS_API fhs_status fhs_measop_dr_cells(fhs_measop* op, int channel, int64_t* cells);
/* Lambda{l}: diag(H)^-1/2 of each data entry of channel l (n_vis(l) values,
 * FP32 precision of the device copy). */
FHS_API fhs_status fhs_measop_dr_lambda(fhs_measop* op, int channel, double* lambda);

/* Autotuner of the operator's launch shapes (no reference counterpart).
 * Candidates, each timed on the operator itself with CUDA events (best of 3
 * after a warm-up): planes per launch of the hand-written real-image FFT
 * passes (all, 16, 8, 4: smaller chunks keep each pass's intermediate in L2
 * for the next), and the most visibilities per gridding work item (8192,
 * 16384, 32768, 65536: dense tiles split into more, shorter items).  The
 * fastest of each is kept for every solver of the operator.  The first
 * fhs_solver_init of an operator runs it unless fhs_measop_set_tuning fixed
 * the shapes.  Split work items sum their partial tiles in another order, so
 * different choices give results that differ at FP32 rounding level; fix the
 * shapes for bit-reproducible runs. */
#define FHS_TUNING_MAX_CANDIDATES 8
typedef struct fhs_tuning {
  int tuned;               /* 1 after fhs_measop_autotune or fhs_measop_set_tuning */
  int fft_chunk;           /* planes per FFT launch (0: all planes; -1: library FFT, not tuned) */
  int grid_slice;          /* visibilities per gridding work item (0: DR operator, not tuned) */
  int n_fft, n_grid;       /* candidates measured (0 when fixed by fhs_measop_set_tuning) */
  int fft_candidates[FHS_TUNING_MAX_CANDIDATES];
  double fft_ms[FHS_TUNING_MAX_CANDIDATES];    /* forward + adjoint transforms, all planes */
  int grid_candidates[FHS_TUNING_MAX_CANDIDATES];
  double grid_ms[FHS_TUNING_MAX_CANDIDATES];   /* whole-operator gridding */
} fhs_tuning;
/* Measure the candidates now and keep the fastest (out may be NULL). */
FHS_API fhs_status fhs_measop_autotune(fhs_measop* op, fhs_tuning* out);
/* Fix the shapes without measuring: fft_chunk >= 0 (0: all planes),
 * grid_slice >= 1024; solvers of op re-capture their iteration graph. */
FHS_API fhs_status fhs_measop_set_tuning(fhs_measop* op, int fft_chunk, int grid_slice);
FHS_API fhs_status fhs_measop_tuning(const fhs_measop* op, fhs_tuning* out);

/* ======================================================================
 * Priors (standalone, device selected per call)
 * ====================================================================== */
/* src/proj_l2ball.m:20-22  p = y + (x-y) min(eps/||x-y||, 1); complex n-vectors, FP64. */
FHS_API fhs_status fhs_proj_l2ball(int device, int64_t n, const double* x, double eps, const double* y,
                           double* p);
/* Allocation-free variant of fhs_proj_l2ball (no counterpart in the
 * reference).  For callers that cannot allocate device memory: hosts whose
 * own pool owns the device heap (MATLAB gpuArray, PyTorch's caching
 * allocator), real-time pipelines that forbid allocation after start-up.  x, y, p are DEVICE pointers to n interleaved
 * complex doubles; the call is enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream) and returns without synchronising.  Scratch: a
 * 512 KB static device array per device that every call shares; n is limited
 * to 134,215,680 (FHS_ERR_UNSUPPORTED above).  The first call on a device
 * (n = 0 is enough) is its set-up: it resolves the array's address
 * (cudaGetSymbolAddress) and loads the call's kernels, so make it before any
 * stream capture.  The resolved address belongs to the device's primary
 * context and is kept for the life of the process: after cudaDeviceReset()
 * on that device, do not call this function again.  Calls that overlap on
 * the GPU (other streams or devices' threads racing on one device) race on
 * the scratch: serialise them. */
FHS_API fhs_status fhs_proj_l2ball_noalloc(int device, int64_t n, const double* x, double eps,
                                           const double* y, double* p, void* stream);
/* src/nuclear_norm.m:25-26  sum of singular values of x reshaped [N, L]. */
FHS_API fhs_status fhs_nuclear_norm(int device, int64_t n_pixels, int L, const double* x, double* f);
/* SARA dictionary (op_p_sp_wlt_basis of the SARA-dictionary submodule,
 * imaging/imaging.m:802): db1..db8 + Dirac, nlevel levels, zero padding,
 * 1/sqrt(9) normalisation.  Coefficients per channel, wavedec2 layout per
 * basis, bases concatenated.  n_coefs returns s (per channel). */
FHS_API int64_t fhs_sara_n_coefs(int Ny, int Nx, int nlevel);
FHS_API fhs_status fhs_sara_analysis(int device, int Ny, int Nx, int L, int nlevel, const double* x,
                             double* coefs);
FHS_API fhs_status fhs_sara_synthesis(int device, int Ny, int Nx, int L, int nlevel, const double* coefs,
                              double* x);
/* src/compute_sara_prior.m:35-41  sum_i ||(Psit x)_i||_2 over channels. */
FHS_API fhs_status fhs_compute_sara_prior(int device, int Ny, int Nx, int L, int nlevel, const double* x,
                                  double* f);

/* ======================================================================
 * Solver: the primal-dual iteration of
 *   facetHyperSARA (src/fhs/facetHyperSARA.m:1-6, loop :701-1138),
 *   hyperSARA      (src/hs/hyperSARA.m:1-3, loop :565-866),
 *   sara           (src/sara/sara.m:1-3, loop :521-837),
 * on the channels of one fhs_measop.  Channels are split into n_groups
 * equal contiguous spectral sub-cubes solved side by side (independent
 * problems: each has its own l21 and nuclear-norm priors and parameters).
 * ====================================================================== */
typedef enum fhs_algo { FHS_ALGO_SARA = 0, FHS_ALGO_HS = 1, FHS_ALGO_FHS = 2 } fhs_algo;
typedef enum fhs_window { FHS_WINDOW_NONE = 0, FHS_WINDOW_TRIANGULAR = 1 } fhs_window;

typedef struct fhs_solver_config {
  int algo;            /* fhs_algo */
  int nlevel;          /* SARA depth (4) */
  int n_groups;        /* spectral sub-cubes, channels per group = L / n_groups */
  int Qy, Qx;          /* spatial facets of the nuclear-norm prior (FHS) */
  const int* splits_y; /* Qy+1 facet boundaries 0..Ny (NULL: split_range) */
  const int* splits_x; /* Qx+1 facet boundaries 0..Nx (NULL: split_range) */
  int overlap_y, overlap_x; /* nuclear-norm facet overlap (pixels) */
  int window;          /* fhs_window (apodisation of the nuclear facets) */
} fhs_solver_config;

/* The `param` fields the solvers read (imaging/imaging.m:839-860,
 * imaging/default_parameters.json).  Arrays: gamma/sig per group,
 * gamma0/sig_bar per group*Q (group-major), nu2 per channel. */
typedef struct fhs_solver_params {
  double nu0, nu1;
  const double* nu2;
  const double* gamma;
  const double* gamma0;
  const double* reweighting_sig;
  const double* reweighting_sig_bar;
  double reweighting_alpha;
  int reweighting_flag;
  int reweighting_min_iter, reweighting_max_iter;
  double reweighting_rel_var;
  int pdfb_min_iter, pdfb_max_iter;
  double pdfb_rel_var, pdfb_fidelity_tolerance, pdfb_rel_var_low;
  /* ellipsoid projection (used when the operator carries a preconditioner);
   * elipse_proj_max_iter <= 0 selects 20 / 1 / 1e-8 for all three */
  int elipse_proj_max_iter, elipse_proj_min_iter;
  double elipse_proj_eps;
  /* noise-level adjustment of fhs_solver_run (facetHyperSARA.m:503-526,
   * 883-951; hyperSARA.m:406-429, 690-737; off in imaging/default_parameters.json):
   * priors off from the run's first iteration until the first adjustment;
   * an adjustment raises eps_b to (eps_b + ||res_b||) change_percentage where
   * eps_b < (2 - pdfb_fidelity_tolerance) ||res_b||, re-estimates the
   * channel noise sigma_l = sqrt(sum_b eps_b^2 / M_l) (the expectation of the
   * reference's randn-based std) and sets gamma = alph sig, gamma0 =
   * alph_bar sig_bar from compute_noise_level.  Values <= 0 select the
   * reference defaults 100 / 1e-3 / 2000 / 0.5 / 1 / 1.  Not used by SARA. */
  int adjust_flag_noise;
  int adjust_noise_min_iter;
  double adjust_noise_rel_var;
  int adjust_noise_start_iter;
  double adjust_noise_change_percentage;
  double alph, alph_bar;
} fhs_solver_params;

/* Per-iteration record (FP64), summed over all groups. */
typedef struct fhs_iter_info {
  double rel_val;         /* sqrt(sum(x-x_prev)^2 / sum x^2) */
  double residual;        /* sqrt(sum_blocks ||G Fx - y||^2) */
  double epsilon;         /* sqrt(sum_blocks eps^2) */
  double nuclear;         /* sum of facet singular values of (v0 + D xhat) before the prox */
} fhs_iter_info;

typedef struct fhs_run_info {
  int n_iter;
  int n_reweights;
  int converged;
  double rel_val, residual, epsilon;
  double seconds;
  int n_noise_adjustments;
} fhs_run_info;

typedef struct fhs_solver fhs_solver;

/* The solver uses op (grids, FFT plans, data layout) on every call: op must
 * outlive every call but the destroy, which touches only the solver's own
 * memory and may come after fhs_measop_destroy. */
FHS_API fhs_status fhs_solver_create(fhs_measop* op, const fhs_solver_config* cfg, fhs_solver** out);
FHS_API fhs_status fhs_solver_destroy(fhs_solver* s);
/* y: visibilities of all channels (whitened, original order); epsilon: one l2
 * bound per block, channel-major. */
FHS_API fhs_status fhs_solver_set_data(fhs_solver* s, const double* y, const double* epsilon);
FHS_API fhs_status fhs_solver_set_params(fhs_solver* s, const fhs_solver_params* p);
/* Initial primal cube x[Ny,Nx,L] (NULL = zeros); initialises duals and
 * weights as fhs_initialize_dual_and_weights.m:88-118 / sara.m:352-362. */
FHS_API fhs_status fhs_solver_init(fhs_solver* s, const double* xinit);
/* n PDFB iterations without stopping test or reweighting (graph replays).
 * info: n records or NULL. */
FHS_API fhs_status fhs_solver_iterate(fhs_solver* s, int n, fhs_iter_info* info);
/* Full solve: iterations, PDFB stopping rule (facetHyperSARA.m:877-881) and
 * reweighting (:952-1137) until convergence or max_iter (<=0: the reference's
 * (reweighting_max_iter+1)*pdfb_max_iter). */
FHS_API fhs_status fhs_solver_run(fhs_solver* s, int max_iter, fhs_run_info* info);
FHS_API fhs_status fhs_solver_get_x(fhs_solver* s, double* x);
/* Forward-backward iterations of the ellipsoid projection in the most recent
 * iteration, one per block (channel-major); all 0 without a preconditioner.
 * The reference's solver_proj_elipse_fb returns the same count as its second
 * output (src/sara/sara.m:561). */
FHS_API fhs_status fhs_solver_ellipse_iterations(fhs_solver* s, int* counts);
/* Current l2 bounds, one per block (channel-major): the values given to
 * set_data, or as adapted by the noise adjustment of fhs_solver_run. */
FHS_API fhs_status fhs_solver_epsilon(fhs_solver* s, double* epsilon);
/* Replaces the l2 bounds (one per block, channel-major) without touching the
 * data: restores adapted bounds from a checkpoint (the reference saves
 * epsilon, facetHyperSARA.m:1071-1107). */
FHS_API fhs_status fhs_solver_set_epsilon(fhs_solver* s, const double* epsilon);
/* Current regularisation parameters gamma[groups] and gamma0[groups x facets]
 * (gamma0 may be NULL; ignored for SARA). */
FHS_API fhs_status fhs_solver_regularization(fhs_solver* s, double* gamma, double* gamma0);

/* Solver state for checkpoints and warm restarts: the arrays the reference
 * saves in its checkpoint files (src/fhs/facetHyperSARA.m:1071-1107: xsol, g,
 * v0, v1, v2, proj, weights0, weights1) and reads back on a warm start
 * (src/fhs/fhs_initialize_dual_and_weights.m, src/sara/sara.m:394-400).
 * Host layouts (doubles, column-major as MATLAB):
 *   X, G       [Ny, Nx, L]
 *   V0         per group, per facet [P_q, lg] (group-major, facets in
 *              column-major facet order), the nuclear-norm duals
 *   V1         [s, L], s = fhs_sara_n_coefs (SARA coefficient layout of
 *              fhs_sara_analysis), the l21 duals
 *   V2, PROJ   all channels' visibilities, interleaved complex, in the
 *              channels' visibility order (PROJ only with a preconditioner)
 *   WEIGHTS0   [lg, Q, n_groups] (group-major: g * Q * lg + q * lg + l)
 *   WEIGHTS1   [s, n_groups]
 * Set fields after fhs_solver_init (which derives the data-term cache from x):
 * the next iteration continues from the restored state. */
typedef enum fhs_field {
  FHS_FIELD_X = 0,
  FHS_FIELD_G = 1,
  FHS_FIELD_V0 = 2,
  FHS_FIELD_V1 = 3,
  FHS_FIELD_V2 = 4,
  FHS_FIELD_PROJ = 5,
  FHS_FIELD_WEIGHTS0 = 6,
  FHS_FIELD_WEIGHTS1 = 7
} fhs_field;
/* doubles of a field in the host layout (0: not present, -1: unknown field) */
FHS_API int64_t fhs_solver_field_size(const fhs_solver* s, int field);
FHS_API fhs_status fhs_solver_get_field(fhs_solver* s, int field, double* out);
FHS_API fhs_status fhs_solver_set_field(fhs_solver* s, int field, const double* in);
/* FP64 statistics of the last iteration, per spectral group (sub-cube):
 * out[g*4 + 0..3] = sum (x - x_prev)^2, sum x^2, sum_b ||G_b Phi x - y_b||^2,
 * sum_b eps_b^2 over the group's channels -- the sums behind rel_val,
 * residual and epsilon of the stopping rule (facetHyperSARA.m:877-881).
 * A caller that splits one cube's sub-cubes over several processes sums
 * them over the processes to take the stopping decision of the whole cube. */
FHS_API fhs_status fhs_solver_group_stats(fhs_solver* s, double* out);
/* Recompute reweighting weights from the current x (fhs_update_weights.m). */
FHS_API fhs_status fhs_solver_update_weights(fhs_solver* s);

/* ======================================================================
 * Learned warm start (no counterpart in the reference; its output is the
 * xinit / varargin{1} of facetHyperSARA.m:1-6, hyperSARA.m:1-3 and
 * sara.m:1-3, used at facetHyperSARA.m:347-350).  A BF16 U-Net (4 levels,
 * 32 base channels, 2,140,065 parameters) maps one normalised dirty image
 * to an initial estimate; trained and run by the library's own kernels.
 * Images are float [n][H][W] (W fastest), H and W multiples of 8; each
 * image is scaled by 1 / max|image| on the way in and its output by the
 * inverse on the way out.  Parameters: a flat float vector, per 3x3 layer
 * (in forward order) weight [Cout][Cin][3][3] then bias [Cout], then the
 * 1x1 head weight [32] and bias [1].
 * ====================================================================== */
typedef struct fhs_unet fhs_unet;
FHS_API fhs_status fhs_unet_create(int device, int base_channels, fhs_unet** out);
FHS_API fhs_status fhs_unet_destroy(fhs_unet* net);
FHS_API int64_t fhs_unet_n_params(const fhs_unet* net);
FHS_API fhs_status fhs_unet_set_params(fhs_unet* net, const float* params);
FHS_API fhs_status fhs_unet_get_params(fhs_unet* net, float* params);
/* out[n][H][W] = network(images) */
FHS_API fhs_status fhs_unet_forward(fhs_unet* net, int n_images, int H, int W, const float* images, float* out);
/* loss = mean((s (out - target))^2) over all pixels (s the image's input
 * scale) and its gradient with respect to every parameter (grad may be NULL) */
FHS_API fhs_status fhs_unet_gradient(fhs_unet* net, int n_images, int H, int W, const float* images,
                                     const float* targets, float* grad, double* loss);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss above */
FHS_API fhs_status fhs_unet_train_step(fhs_unet* net, int n_images, int H, int W, const float* images,
                                       const float* targets, float lr, double* loss);
/* fhs_solver_init from the learned warm start, on the device (no cube
 * crosses to the host): the normalised dirty cube Re(Phi^H y) / PSF peak per
 * channel (src/compute_residual_images.m:83-102 at x = 0) from the solver's
 * operator and data, the network on every channel (chunk images per batch,
 * <= 0: 16), clipped at 0, then the fallback rule: the solver starts from
 * that estimate x0 if F(x0) < F(0), else from zero, with
 *   F(x) = sum_b max(0, ||y_b - Phi_b x|| - eps_b)
 *          + sum_g gamma_g ||Psi^T x_g||_{2,1} + sum_g gamma0_g ||x_g||_*
 * (the nuclear term for the FHS / HS priors, over each whole spectral
 * sub-cube with the group's first facet weight).  Needs set_data and
 * set_params, a visibility (not DR) operator, image sides divisible by 8,
 * and the network on the solver's device.  info may be NULL. */
typedef struct fhs_warm_info {
  int used;               /* 1: the solver starts from the network's estimate */
  double objective_warm;  /* F(x0) */
  double objective_cold;  /* F(0) */
  double seconds;         /* host wall time of the call, initialisation included */
} fhs_warm_info;
FHS_API fhs_status fhs_solver_init_warm(fhs_solver* s, fhs_unet* net, int chunk, fhs_warm_info* info);

/* Measurement hooks (no reference counterpart: the reference times its
 * phases with tic/toc, src/fhs/facetHyperSARA.m:703-716,771-776).
 * time_iterations: n graph replays bracketed by CUDA events on the solver's
 * stream, total device milliseconds.  profile_stages: n iterations launched
 * stage by stage with events in between, mean milliseconds per stage. */
FHS_API int fhs_solver_stage_count(void);
FHS_API const char* fhs_solver_stage_name(int i);
FHS_API fhs_status fhs_solver_time_iterations(fhs_solver* s, int n, double* ms);
FHS_API fhs_status fhs_solver_profile_stages(fhs_solver* s, int n, double* stage_ms);

#ifdef __cplusplus
}
#endif

#endif /* FHS_B200_H */
