// Primal-dual solver state and iteration (see solver.cu).
#pragma once

#include "measop.cuh"
#include "nuclear.cuh"
#include "sara.cuh"

namespace fhs {

constexpr int kReportFields = 6;   // rel_x, norm_x, res^2, eps^2, nuclear, l21 (per group)
constexpr int kReportRing = 1024;  // iterations kept on the device between host reads

struct Solver {
  MeasOp* op = nullptr;
  int device = 0;               // op->device, kept so that destroy never reads op
  int algo = FHS_ALGO_FHS, nlevel = 4, G = 1, lg = 1, L = 1, Ny = 0, Nx = 0;
  int64_t N = 0;
  SaraPlan sp;
  NucPlan np;
  bool nuclear = true;

  DevBuf<float> x, g, xhat, g1, coef, apx, v1, w1, v0, rownorm;
  DevBuf<double> beta1, w0, beta0, sig_bar, sig;
  DevBuf<float2> y, v2, gold;
  DevBuf<double2> projw;        // proj - y of the ellipsoid projection (preconditioned operator)
  bool precond = false;         // operator carried a preconditioner at init
  int fb_max = 20, fb_min = 1;  // elipse_proj_max_iter / min_iter
  double fb_stop = 1e-8;        // elipse_proj_eps
  DevBuf<float> sigma22;
  DevBuf<double> primal_part;   // [L][kPrimalBlocks][2]
  DevBuf<double> l21_part;      // [G][prox blocks] (unfused prox path)
  DevBuf<double> l21_acc;       // [G] sum of row norms (fused path)
  DevBuf<double> nuc_vals;      // [G][Q]
  DevBuf<double> ring;          // [kReportRing][G][kReportFields]
  DevBuf<int> ring_counter;
  int prox_blocks = 0;

  // parameters (host)
  double tau = 0, sigma00 = 0, sigma11 = 0;
  std::vector<double> nu2, gamma, gamma0, rw_sig, rw_sig_bar;
  double rw_alpha = 1.0;
  int rw_flag = 1, rw_min = 1, rw_max = 20;
  double rw_rel_var = 1e-4;
  int pdfb_min = 10, pdfb_max = 2000;
  double pdfb_rel_var = 5e-5, pdfb_tol = 1.01, pdfb_rel_var_low = 5e-6;
  double sigma0 = 1.0, sigma1 = 1.0;
  // noise-level adjustment (fhs_solver_run)
  bool adjust_noise = false;
  int adjust_min_iter = 100, adjust_start_iter = 2000;
  double adjust_rel_var = 1e-3, adjust_change = 0.5, alph = 1.0, alph_bar = 1.0;
  std::vector<double> h_eps;     // [nblk_tot] current l2 bounds
  bool params_set = false, data_set = false, initialised = false;

  cudaGraphExec_t graph = nullptr;
  int graph_epoch = -1;   // op->layout_epoch the graph was captured at
  unsigned long long launches_per_iter = 0;
  long long iter_done = 0;       // iterations since init
  long long ring_read = 0;       // iterations already read back
  ~Solver();
};

// fhs_solver_init from a host FP64 cube, a device FP32 cube [L][Nx][Ny]
// (xinit_dev), or zeros (both NULL)
void solver_init_state(Solver* S, const double* xinit, const float* xinit_dev);

}  // namespace fhs
