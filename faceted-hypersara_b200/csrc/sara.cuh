// SARA dictionary on the device: db1..db8 + Dirac, zero padding (see sara.cu).
#pragma once

#include "common.cuh"

namespace fhs {

constexpr int kSaraWavelets = 8;   // db1..db8
constexpr int kSaraMaxLevel = 8;
constexpr int kSaraMaxFilter = 16;

// Geometry of the SARA coefficient vector of one channel (wavedec2 layout per
// basis, bases concatenated, Dirac last) and of the intermediate
// approximation planes.
struct SaraPlan {
  int Ny = 0, Nx = 0, J = 0;
  int n0[kSaraWavelets][kSaraMaxLevel + 1];  // level sizes along y (level 0 = image)
  int n1[kSaraWavelets][kSaraMaxLevel + 1];  // along x
  int64_t offA[kSaraWavelets];                         // A_J inside the channel vector
  int64_t offH[kSaraWavelets][kSaraMaxLevel + 1];      // H_j (j = 1..J); V_j, D_j follow
  int64_t boff[kSaraWavelets + 1];                     // basis starts (Dirac = boff[8])
  int64_t s = 0;                                       // coefficients per channel
  int64_t apx_off[kSaraWavelets][kSaraMaxLevel + 1];   // approximation planes, levels 1..J-1
  int64_t apx_total = 0;                               // approximation floats per channel
};

SaraPlan sara_plan(int Ny, int Nx, int J);

// Analysis Psit of planes [0, np) of `x` (plane stride Ny*Nx) into `coef`
// (plane stride plan.s); the Dirac part is left untouched (it equals x/3).
// `apx`: scratch of np * plan.apx_total floats.
void sara_analysis(const SaraPlan& p, const float* x, float* coef, float* apx, int np, cudaStream_t s);
// Synthesis Psi of `coef` (all bases including Dirac) into out = alpha * Psi(coef).
void sara_synthesis(const SaraPlan& p, const float* coef, float* out, float* apx, int np, float alpha,
                    cudaStream_t s);
// Dirac part of the analysis: coef[:, boff[8]:] = x / 3.
void sara_dirac(const SaraPlan& p, const float* x, float* coef, int np, cudaStream_t s);

// Weighted l21 prox of the dual (fhs_update_dual_sparsity.m:84-89) for
// groups of lg consecutive planes: w = v1 + coef (Dirac part: v1 + xhat/3),
// l2 over the group, v1 <- w - max(l2 - beta*weights, 0)/(l2 + eps) * w.
// weights: [n_groups][s]; beta: [n_groups] (device).  xhat: image planes.
// l21 (optional, [n_groups] FP64): sum over coefficients of l2.
void sara_l21_prox(const SaraPlan& p, float* v1, const float* coef, const float* xhat, const float* weights,
                   const double* beta, int n_groups, int lg, double* l21_partials, cudaStream_t s);
// Fused analysis + weighted l21 prox of every level and of the Dirac part
// (coefficients never written): v1 <- prox(v1 + Psit xhat) per group of lg
// (<= 32) channels.  l21_acc[g] (FP64, zeroed by the caller) receives
// sum_i ||v1_i + (Psit xhat)_i||_2.
bool sara_fused_supported(int lg);
void sara_analysis_prox(const SaraPlan& p, const float* xhat, float* v1, float* apx, const float* weights,
                        const double* beta, int n_groups, int lg, double* l21_acc, cudaStream_t s);
// Row l2 norms over a group of the analysis coefficients (coef + Dirac from
// x): out[g][i] = ||coef_i||.  Used for weights and prior values.
void sara_row_norms(const SaraPlan& p, const float* coef, const float* x, int n_groups, int lg, float* out,
                    cudaStream_t s);

}  // namespace fhs
