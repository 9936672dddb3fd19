/*
 * fhs_mex.c -- MATLAB MEX gateway over the libfhs_b200 C ABI.
 *
 *   mex -R2018a fhs_mex.c -I<repo>/include -L<repo>/faceted-hypersara_b200/fhs_b200 -lfhs_b200
 *
 * One command string per entry point; handles travel as uint64 scalars.
 * Complex arrays use MATLAB's interleaved storage (R2018a API), which is the
 * ABI's layout, so no copies are made on the way in.  The reference's MATLAB
 * signatures are kept by thin .m wrappers, e.g.
 *   y  = apply_direct_operator(Fx, G, Lambda)   ->  fhs_mex('apply_direct_operator', G.h, G.channel, Fx)
 *   xsol = facetHyperSARA(y, epsilon, A, At, pU, G, W, param, Qx, Qy, ...)
 *        ->  fhs_mex('solver', G.h, 'fhs', cfg, param, cat(1, y{:}{:}), cat(1, epsilon{:}{:}), xinit)
 *
 * Commands (inputs after the command string -> outputs):
 *   measop_create       Ny, Nx, oy, ox, J, L, device            -> h
 *   measop_set_channel  h, l, om_y, om_x, weights|[], blocks    -> -
 *   measop_commit       h                                       -> -
 *   measop_destroy      h                                       -> -
 *   measop_create_dr    h                                       -> h_dr
 *   measop_set_preconditioner  h, l, pU                         -> -
 *   measop_n_vis        h, l                                    -> n
 *   apply_direct_operator      h, l, Fx                         -> y
 *   apply_adjoint_operator     h, l, y                          -> Fx
 *   HS_forward_operator_G      h, x                             -> y (all channels)
 *   HS_adjoint_operator_G      h, y, [Ny Nx L]                  -> x
 *   operator_norm       h, max_iter, tol, L                     -> nu2
 *   update_dual_data_fidelity  h, v2, y, x, Fx_old, epsilon, sigma22
 *                                  -> v2, Ftx, Fx_old, norm_res, global_norm_res, norm_epsilon
 *   update_dual_data_fidelity_precond  h, v2, proj, y, x, Fx_old, epsilon,
 *                                  elipse_proj_max_iter, elipse_proj_min_iter, elipse_proj_eps, sigma22
 *                                  -> v2, Ftx, Fx_old, proj, norm_res, global_norm_res, norm_epsilon
 *   proj_l2ball         x, eps, y                               -> p
 *   nuclear_norm        x [N, L]                                -> f
 *   compute_sara_prior  x [Ny, Nx, L], nlevel                   -> f
 *   solver              h, algo, cfg, param, y, epsilon, xinit|[] -> xsol, info
 */
#include <stdint.h>
#include <string.h>

#include "fhs_b200.h"
#include "mex.h"

static void check(fhs_status s) {
  if (s != FHS_OK) mexErrMsgIdAndTxt("fhs:error", "%s", fhs_last_error());
}

static void need(int ok, const char* msg) {
  if (!ok) mexErrMsgIdAndTxt("fhs:usage", "%s", msg);
}

static fhs_measop* op_of(const mxArray* a) {
  need(mxGetClassID(a) == mxUINT64_CLASS && mxGetNumberOfElements(a) == 1, "expected an operator handle");
  return (fhs_measop*)(uintptr_t)(*(uint64_t*)mxGetData(a));
}

static mxArray* handle_out(void* p) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  *(uint64_t*)mxGetData(a) = (uint64_t)(uintptr_t)p;
  return a;
}

static const double* cplx_in(const mxArray* a) {
  need(mxIsDouble(a) && mxIsComplex(a), "expected a complex double array");
  return (const double*)mxGetComplexDoubles(a);
}

static const double* real_in(const mxArray* a) {
  need(mxIsDouble(a) && !mxIsComplex(a), "expected a real double array");
  return mxGetDoubles(a);
}

static double field_num(const mxArray* s, const char* name, double dflt) {
  const mxArray* f = mxIsStruct(s) ? mxGetField(s, 0, name) : NULL;
  return f && !mxIsEmpty(f) ? mxGetScalar(f) : dflt;
}

static const double* field_arr(const mxArray* s, const char* name, size_t n) {
  const mxArray* f = mxIsStruct(s) ? mxGetField(s, 0, name) : NULL;
  need(f && mxIsDouble(f) && mxGetNumberOfElements(f) >= n, name);
  return mxGetDoubles(f);
}

static int64_t total_vis(fhs_measop* op, int L) {
  int64_t n = 0;
  for (int l = 0; l < L; ++l) n += fhs_measop_n_vis(op, l);
  return n;
}

/* Sizes every operand of an operator call must have: the library reads and
 * writes exactly these counts, so a short MATLAB array is a usage error here
 * instead of a heap overrun inside the MATLAB process. */
typedef struct {
  int Ny, Nx, L;
  int64_t n_vis;   /* all channels */
  int64_t n_blk;   /* all channels */
  int64_t No;
} op_shape;

static op_shape shape_of(fhs_measop* op) {
  op_shape sh;
  memset(&sh, 0, sizeof sh);
  check(fhs_measop_image_size(op, &sh.Ny, &sh.Nx, &sh.L));
  for (int l = 0; l < sh.L; ++l) {
    sh.n_vis += fhs_measop_n_vis(op, l);
    sh.n_blk += fhs_measop_n_blocks(op, l);
  }
  sh.No = fhs_measop_grid_size(op);
  return sh;
}

static void need_numel(const mxArray* a, int64_t n, const char* msg) {
  need((int64_t)mxGetNumberOfElements(a) == n, msg);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[64];
  need(nrhs >= 1 && mxIsChar(prhs[0]) && mxGetString(prhs[0], cmd, sizeof cmd) == 0, "first input: command");
  if (!strcmp(cmd, "measop_create")) {
    need(nrhs == 8, "measop_create(Ny, Nx, oy, ox, J, L, device)");
    fhs_measop* op = NULL;
    const int J = (int)mxGetScalar(prhs[5]);
    check(fhs_measop_create((int)mxGetScalar(prhs[7]), (int)mxGetScalar(prhs[1]), (int)mxGetScalar(prhs[2]),
                            (int)mxGetScalar(prhs[3]), (int)mxGetScalar(prhs[4]), J, J,
                            (int)mxGetScalar(prhs[6]), &op));
    plhs[0] = handle_out(op);
  } else if (!strcmp(cmd, "measop_set_channel")) {
    need(nrhs == 7, "measop_set_channel(h, l, om_y, om_x, weights, blocks)");
    const mwSize n = mxGetNumberOfElements(prhs[3]);
    const mwSize nb = mxGetNumberOfElements(prhs[6]);
    need(nb >= 1 && nb <= 16, "1 to 16 blocks");
    need(mxGetNumberOfElements(prhs[4]) == n, "om_x: same size as om_y");
    need(mxIsEmpty(prhs[5]) || mxGetNumberOfElements(prhs[5]) == n, "weights: [] or one per visibility");
    int64_t bs[16];
    const double* b = real_in(prhs[6]);
    for (mwSize k = 0; k < nb; ++k) bs[k] = (int64_t)b[k];
    check(fhs_measop_set_channel(op_of(prhs[1]), (int)mxGetScalar(prhs[2]), (int64_t)n, real_in(prhs[3]),
                                 real_in(prhs[4]), mxIsEmpty(prhs[5]) ? NULL : real_in(prhs[5]), (int)nb, bs));
  } else if (!strcmp(cmd, "measop_commit")) {
    check(fhs_measop_commit(op_of(prhs[1])));
  } else if (!strcmp(cmd, "measop_destroy")) {
    check(fhs_measop_destroy(op_of(prhs[1])));
  } else if (!strcmp(cmd, "measop_create_dr")) {
    fhs_measop* dr = NULL;
    check(fhs_measop_create_dr(op_of(prhs[1]), &dr));
    plhs[0] = handle_out(dr);
  } else if (!strcmp(cmd, "measop_set_preconditioner")) {
    need(nrhs == 4, "measop_set_preconditioner(h, l, pU)");
    fhs_measop* op = op_of(prhs[1]);
    const int ch = (int)mxGetScalar(prhs[2]);
    need(fhs_measop_n_vis(op, ch) >= 0, "channel out of range");
    need_numel(prhs[3], fhs_measop_n_vis(op, ch), "pU: one entry per visibility of the channel");
    check(fhs_measop_set_preconditioner(op, ch, real_in(prhs[3])));
  } else if (!strcmp(cmd, "measop_n_vis")) {
    plhs[0] = mxCreateDoubleScalar((double)fhs_measop_n_vis(op_of(prhs[1]), (int)mxGetScalar(prhs[2])));
  } else if (!strcmp(cmd, "apply_direct_operator")) { /* src/apply_direct_operator.m:1 */
    need(nrhs == 4, "apply_direct_operator(h, l, Fx)");
    fhs_measop* op = op_of(prhs[1]);
    const int ch = (int)mxGetScalar(prhs[2]);
    need(fhs_measop_n_vis(op, ch) >= 0, "channel out of range");
    need_numel(prhs[3], fhs_measop_grid_size(op), "Fx: one entry per grid point (No = Ky*Kx)");
    plhs[0] = mxCreateDoubleMatrix((mwSize)fhs_measop_n_vis(op, ch), 1, mxCOMPLEX);
    check(fhs_apply_direct_operator(op, ch, cplx_in(prhs[3]), (double*)mxGetComplexDoubles(plhs[0])));
  } else if (!strcmp(cmd, "apply_adjoint_operator")) { /* src/apply_adjoint_operator.m:1 */
    need(nrhs == 4, "apply_adjoint_operator(h, l, y)");
    fhs_measop* op = op_of(prhs[1]);
    const int ch = (int)mxGetScalar(prhs[2]);
    need(fhs_measop_n_vis(op, ch) >= 0, "channel out of range");
    need_numel(prhs[3], fhs_measop_n_vis(op, ch), "y: one entry per visibility of the channel");
    plhs[0] = mxCreateDoubleMatrix((mwSize)fhs_measop_grid_size(op), 1, mxCOMPLEX);
    check(fhs_apply_adjoint_operator(op, (int)mxGetScalar(prhs[2]), cplx_in(prhs[3]),
                                     (double*)mxGetComplexDoubles(plhs[0])));
  } else if (!strcmp(cmd, "HS_forward_operator_G")) { /* lib/operators/HS_forward_operator_G.m */
    need(nrhs == 3, "HS_forward_operator_G(h, x)");
    fhs_measop* op = op_of(prhs[1]);
    const op_shape sh = shape_of(op);
    need_numel(prhs[2], (int64_t)sh.Ny * sh.Nx * sh.L, "x: [Ny, Nx, L] of the operator");
    plhs[0] = mxCreateDoubleMatrix((mwSize)total_vis(op, sh.L), 1, mxCOMPLEX);
    check(fhs_forward_operator(op, real_in(prhs[2]), (double*)mxGetComplexDoubles(plhs[0])));
  } else if (!strcmp(cmd, "HS_adjoint_operator_G")) { /* lib/operators/HS_adjoint_operator_G.m, then real() */
    need(nrhs == 4, "HS_adjoint_operator_G(h, y, [Ny Nx L])");
    fhs_measop* op = op_of(prhs[1]);
    need(mxGetNumberOfElements(prhs[3]) == 3, "cube size [Ny Nx L]");
    const double* sz = real_in(prhs[3]);
    const op_shape sh = shape_of(op);
    need(sz[0] == sh.Ny && sz[1] == sh.Nx && sz[2] == sh.L, "cube size [Ny Nx L] of the operator");
    need_numel(prhs[2], sh.n_vis, "y: all channels' visibilities");
    const mwSize dims[3] = {(mwSize)sz[0], (mwSize)sz[1], (mwSize)sz[2]};
    plhs[0] = mxCreateNumericArray(3, dims, mxDOUBLE_CLASS, mxREAL);
    check(fhs_adjoint_operator(op, cplx_in(prhs[2]), mxGetDoubles(plhs[0])));
  } else if (!strcmp(cmd, "operator_norm")) { /* lib/utils/util_operator_norm.m */
    need(nrhs == 5, "operator_norm(h, max_iter, tol, L)");
    fhs_measop* op = op_of(prhs[1]);
    const int L = (int)mxGetScalar(prhs[4]);
    need(L == shape_of(op).L, "L: the operator's channel count");
    plhs[0] = mxCreateDoubleMatrix((mwSize)L, 1, mxREAL);
    check(fhs_operator_norm(op, (int)mxGetScalar(prhs[2]), mxGetScalar(prhs[3]), mxGetDoubles(plhs[0])));
  } else if (!strcmp(cmd, "update_dual_data_fidelity")) { /* src/update_dual_data_fidelity.m:1-6 */
    need(nrhs == 8, "update_dual_data_fidelity(h, v2, y, x, Fx_old, epsilon, sigma22)");
    fhs_measop* op = op_of(prhs[1]);
    const mwSize* d = mxGetDimensions(prhs[4]);
    (void)cplx_in(prhs[2]);  /* v2 and Fx_old must be complex (usage error otherwise) */
    (void)cplx_in(prhs[5]);
    {
      const op_shape sh = shape_of(op);
      need_numel(prhs[2], sh.n_vis, "v2: all channels' visibilities");
      need_numel(prhs[3], sh.n_vis, "y: all channels' visibilities");
      need_numel(prhs[4], (int64_t)sh.Ny * sh.Nx * sh.L, "x: [Ny, Nx, L] of the operator");
      need_numel(prhs[5], sh.No * sh.L, "Fx_old: [No, L]");
      need_numel(prhs[6], sh.n_blk, "epsilon: one bound per block");
      need_numel(prhs[7], sh.L, "sigma22: one per channel");
    }
    mxArray* out[6];
    out[0] = mxDuplicateArray(prhs[2]);                                    /* v2 (updated) */
    out[1] = mxCreateNumericArray(mxGetNumberOfDimensions(prhs[4]), d, mxDOUBLE_CLASS, mxREAL);  /* Ftx */
    out[2] = mxDuplicateArray(prhs[5]);                                    /* Fx_old (updated) */
    out[3] = mxCreateDoubleMatrix(mxGetNumberOfElements(prhs[6]), 1, mxREAL); /* norm_res per block */
    out[4] = mxCreateDoubleScalar(0.0);
    out[5] = mxCreateDoubleScalar(0.0);
    const fhs_status st = fhs_update_dual_data_fidelity(
        op, (double*)mxGetComplexDoubles(out[0]), cplx_in(prhs[3]), real_in(prhs[4]),
        (double*)mxGetComplexDoubles(out[2]), real_in(prhs[6]), real_in(prhs[7]), mxGetDoubles(out[1]),
        mxGetDoubles(out[3]), mxGetDoubles(out[4]), mxGetDoubles(out[5]));
    /* plhs holds max(nlhs, 1) entries: hand over the requested outputs only */
    for (int k = 0; k < 6; ++k) {
      if (k < nlhs || k == 0)
        plhs[k] = out[k];
      else
        mxDestroyArray(out[k]);
    }
    check(st);
  } else if (!strcmp(cmd, "update_dual_data_fidelity_precond")) { /* src/update_dual_data_fidelity.m:126-147 */
    need(nrhs == 12, "update_dual_data_fidelity_precond(h, v2, proj, y, x, Fx_old, epsilon, "
                     "elipse_proj_max_iter, elipse_proj_min_iter, elipse_proj_eps, sigma22)");
    fhs_measop* op = op_of(prhs[1]);
    const mwSize* d = mxGetDimensions(prhs[5]);
    (void)cplx_in(prhs[2]);  /* v2, proj and Fx_old must be complex (usage error otherwise) */
    (void)cplx_in(prhs[3]);
    (void)cplx_in(prhs[6]);
    {
      const op_shape sh = shape_of(op);
      need_numel(prhs[2], sh.n_vis, "v2: all channels' visibilities");
      need_numel(prhs[3], sh.n_vis, "proj: all channels' visibilities");
      need_numel(prhs[4], sh.n_vis, "y: all channels' visibilities");
      need_numel(prhs[5], (int64_t)sh.Ny * sh.Nx * sh.L, "x: [Ny, Nx, L] of the operator");
      need_numel(prhs[6], sh.No * sh.L, "Fx_old: [No, L]");
      need_numel(prhs[7], sh.n_blk, "epsilon: one bound per block");
      need_numel(prhs[11], sh.L, "sigma22: one per channel");
    }
    mxArray* out[7];
    out[0] = mxDuplicateArray(prhs[2]);                                    /* v2 (updated) */
    out[1] = mxCreateNumericArray(mxGetNumberOfDimensions(prhs[5]), d, mxDOUBLE_CLASS, mxREAL);  /* Ftx */
    out[2] = mxDuplicateArray(prhs[6]);                                    /* Fx_old (updated) */
    out[3] = mxDuplicateArray(prhs[3]);                                    /* proj (updated) */
    out[4] = mxCreateDoubleMatrix(mxGetNumberOfElements(prhs[7]), 1, mxREAL); /* norm_res per block */
    out[5] = mxCreateDoubleScalar(0.0);
    out[6] = mxCreateDoubleScalar(0.0);
    const fhs_status st = fhs_update_dual_data_fidelity_precond(
        op, (double*)mxGetComplexDoubles(out[0]), (double*)mxGetComplexDoubles(out[3]), cplx_in(prhs[4]),
        real_in(prhs[5]), (double*)mxGetComplexDoubles(out[2]), real_in(prhs[7]), (int)mxGetScalar(prhs[8]),
        (int)mxGetScalar(prhs[9]), mxGetScalar(prhs[10]), real_in(prhs[11]), mxGetDoubles(out[1]),
        mxGetDoubles(out[4]), mxGetDoubles(out[5]), mxGetDoubles(out[6]), NULL);
    for (int k = 0; k < 7; ++k) {
      if (k < nlhs || k == 0)
        plhs[k] = out[k];
      else
        mxDestroyArray(out[k]);
    }
    check(st);
  } else if (!strcmp(cmd, "proj_l2ball")) { /* src/proj_l2ball.m:1 */
    need(nrhs == 4, "proj_l2ball(x, eps, y)");
    const mwSize n = mxGetNumberOfElements(prhs[1]);
    need(mxGetNumberOfElements(prhs[3]) == n, "y: same size as x");
    plhs[0] = mxCreateDoubleMatrix(n, 1, mxCOMPLEX);
    check(fhs_proj_l2ball(0, (int64_t)n, cplx_in(prhs[1]), mxGetScalar(prhs[2]), cplx_in(prhs[3]),
                          (double*)mxGetComplexDoubles(plhs[0])));
  } else if (!strcmp(cmd, "nuclear_norm")) { /* src/nuclear_norm.m:1 */
    double f = 0.0;
    check(fhs_nuclear_norm(0, (int64_t)mxGetM(prhs[1]), (int)mxGetN(prhs[1]), real_in(prhs[1]), &f));
    plhs[0] = mxCreateDoubleScalar(f);
  } else if (!strcmp(cmd, "compute_sara_prior")) { /* src/compute_sara_prior.m:1 */
    const mwSize* d = mxGetDimensions(prhs[1]);
    const int L = mxGetNumberOfDimensions(prhs[1]) > 2 ? (int)d[2] : 1;
    double f = 0.0;
    check(fhs_compute_sara_prior(0, (int)d[0], (int)d[1], L, (int)mxGetScalar(prhs[2]), real_in(prhs[1]), &f));
    plhs[0] = mxCreateDoubleScalar(f);
  } else if (!strcmp(cmd, "solver")) {
    /* facetHyperSARA.m:1-6 / hyperSARA.m:1-3 / sara.m:1-3 through the solver
     * handle: solver(h, algo, cfg, param, y, epsilon, xinit) -> xsol, info */
    need(nrhs == 8, "solver(h, algo, cfg, param, y, epsilon, xinit)");
    fhs_measop* op = op_of(prhs[1]);
    char algo[8];
    mxGetString(prhs[2], algo, sizeof algo);
    const mxArray* cfg_s = prhs[3];
    const mxArray* par = prhs[4];
    fhs_solver_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.algo = !strcmp(algo, "sara") ? FHS_ALGO_SARA : !strcmp(algo, "hs") ? FHS_ALGO_HS : FHS_ALGO_FHS;
    cfg.nlevel = (int)field_num(cfg_s, "nlevel", 4);
    cfg.n_groups = (int)field_num(cfg_s, "n_groups", 1);
    cfg.Qy = (int)field_num(cfg_s, "Qy", 1);
    cfg.Qx = (int)field_num(cfg_s, "Qx", 1);
    cfg.overlap_y = (int)field_num(cfg_s, "overlap_y", 0);
    cfg.overlap_x = (int)field_num(cfg_s, "overlap_x", 0);
    cfg.window = (int)field_num(cfg_s, "window", cfg.algo == FHS_ALGO_FHS ? FHS_WINDOW_TRIANGULAR : FHS_WINDOW_NONE);
    const int L = (int)field_num(cfg_s, "L", 1);
    {
      const op_shape sh = shape_of(op);
      need(L == sh.L && (int)field_num(cfg_s, "Ny", 0) == sh.Ny && (int)field_num(cfg_s, "Nx", 0) == sh.Nx,
           "cfg.Ny, cfg.Nx, cfg.L: the operator's image size and channel count");
      need_numel(prhs[5], sh.n_vis, "y: all channels' visibilities");
      need_numel(prhs[6], sh.n_blk, "epsilon: one bound per block");
      need(mxIsEmpty(prhs[7]) || (int64_t)mxGetNumberOfElements(prhs[7]) == (int64_t)sh.Ny * sh.Nx * sh.L,
           "xinit: [] or [Ny, Nx, L]");
    }
    const int G = cfg.algo == FHS_ALGO_SARA ? L : cfg.n_groups;
    const int Q = cfg.algo == FHS_ALGO_FHS ? cfg.Qy * cfg.Qx : 1;
    fhs_solver_params p;
    memset(&p, 0, sizeof p);
    p.nu0 = field_num(par, "nu0", 1.0);
    p.nu1 = field_num(par, "nu1", 1.0);
    p.nu2 = field_arr(par, "nu2", (size_t)L);
    p.gamma = field_arr(par, "gamma", (size_t)G);
    p.reweighting_sig = field_arr(par, "reweighting_sig", (size_t)G);
    if (cfg.algo != FHS_ALGO_SARA) {
      p.gamma0 = field_arr(par, "gamma0", (size_t)G * Q);
      p.reweighting_sig_bar = field_arr(par, "reweighting_sig_bar", (size_t)G * Q);
    }
    p.reweighting_alpha = field_num(par, "reweighting_alpha", 1.0);
    p.reweighting_flag = (int)field_num(par, "reweighting_flag", 1);
    p.reweighting_min_iter = (int)field_num(par, "reweighting_min_iter", 1);
    p.reweighting_max_iter = (int)field_num(par, "reweighting_max_iter", 20);
    p.reweighting_rel_var = field_num(par, "reweighting_rel_var", 1e-4);
    p.pdfb_min_iter = (int)field_num(par, "pdfb_min_iter", 10);
    p.pdfb_max_iter = (int)field_num(par, "pdfb_max_iter", 2000);
    p.pdfb_rel_var = field_num(par, "pdfb_rel_var", 5e-5);
    p.pdfb_fidelity_tolerance = field_num(par, "pdfb_fidelity_tolerance", 1.01);
    p.pdfb_rel_var_low = field_num(par, "pdfb_rel_var_low", 5e-6);
    p.elipse_proj_max_iter = (int)field_num(par, "elipse_proj_max_iter", 20);
    p.elipse_proj_min_iter = (int)field_num(par, "elipse_proj_min_iter", 1);
    p.elipse_proj_eps = field_num(par, "elipse_proj_eps", 1e-8);
    p.adjust_flag_noise = (int)field_num(par, "adjust_flag_noise", 0);
    p.adjust_noise_min_iter = (int)field_num(par, "adjust_noise_min_iter", 100);
    p.adjust_noise_rel_var = field_num(par, "adjust_noise_rel_var", 1e-3);
    p.adjust_noise_start_iter = (int)field_num(par, "adjust_noise_start_iter", 2000);
    p.adjust_noise_change_percentage = field_num(par, "adjust_noise_change_percentage", 0.5);
    p.alph = field_num(par, "alph", 1.0);
    p.alph_bar = field_num(par, "alph_bar", 1.0);
    fhs_solver* s = NULL;
    check(fhs_solver_create(op, &cfg, &s));
    fhs_status st = fhs_solver_set_params(s, &p);
    if (st == FHS_OK) st = fhs_solver_set_data(s, cplx_in(prhs[5]), real_in(prhs[6]));
    if (st == FHS_OK) st = fhs_solver_init(s, mxIsEmpty(prhs[7]) ? NULL : real_in(prhs[7]));
    fhs_run_info ri;
    memset(&ri, 0, sizeof ri);
    if (st == FHS_OK) st = fhs_solver_run(s, 0, &ri);
    const mwSize dims[3] = {(mwSize)field_num(cfg_s, "Ny", 0), (mwSize)field_num(cfg_s, "Nx", 0), (mwSize)L};
    plhs[0] = mxCreateNumericArray(3, dims, mxDOUBLE_CLASS, mxREAL);
    if (st == FHS_OK) st = fhs_solver_get_x(s, mxGetDoubles(plhs[0]));
    fhs_solver_destroy(s);
    check(st);
    if (nlhs > 1) { /* info = [n_iter, n_reweights, converged, rel_val, residual, seconds] */
      plhs[1] = mxCreateDoubleMatrix(1, 6, mxREAL);
      double* o = mxGetDoubles(plhs[1]);
      o[0] = ri.n_iter;
      o[1] = ri.n_reweights;
      o[2] = ri.converged;
      o[3] = ri.rel_val;
      o[4] = ri.residual;
      o[5] = ri.seconds;
    }
  } else {
    mexErrMsgIdAndTxt("fhs:usage", "unknown command '%s'", cmd);
  }
}
