// Faceted nuclear-norm prior on the device (see nuclear.cu).
#pragma once

#include "common.cuh"

namespace fhs {

constexpr int kNucMaxL = 64;       // channels per spectral group
constexpr int kNucChunk = 2048;    // pixels per Gram / reconstruction CTA

struct NucFacet {
  int y0, y1, x0, x1;     // overlapped facet [y0, y1) x [x0, x1)
  int64_t v0_off;         // offset of the facet's dual inside a group's block ([lg][P])
  int64_t wy_off, wx_off; // offsets of its 1-D windows
  int nchunks;            // ceil(P / kNucChunk)
};

struct NucPlan {
  int Ny = 0, Nx = 0, Qy = 0, Qx = 0, Q = 0, n_groups = 0, lg = 0;
  std::vector<NucFacet> facets;
  int max_chunks = 0;
  int64_t v0_group = 0;      // floats of v0 per group (lg * sum_q P_q)
  DevBuf<NucFacet> d_facets;
  DevBuf<float> wy, wx;      // concatenated windows
  DevBuf<int> cover_y, cover_x;  // [N][2] facet index along the axis or -1
  DevBuf<float> gram_part;   // [G][Q][max_chunks][lg*lg]
  DevBuf<double> gram;       // [G][Q][lg][lg]
  DevBuf<float> shrinkM;     // [G][Q][lg][lg]  M = I - V diag(shrink) V^T
  DevBuf<double> sigma;      // [G][Q][lg] singular values (descending)
};

// Facet geometry: splits (Qy+1 / Qx+1 boundaries), overlap towards lower
// indices, triangular or flat windows (see window_1d below).
void nuc_plan_init(NucPlan& p, int Ny, int Nx, int Qy, int Qx, const std::vector<int>& splits_y,
                   const std::vector<int>& splits_x, int overlap_y, int overlap_x, int window, int n_groups,
                   int lg, cudaStream_t s);

// Gram_q = Z^T Z with Z = v0_q + D_q .* xhat_q (v0 may be null = 0).
void nuc_gram(const NucPlan& p, const float* xhat, const float* v0, cudaStream_t s);
// Gram of one FP64 [lg][N] matrix in FP64 (n_groups = Q = 1 plans), into p.gram.
void nuc_gram_fp64(const NucPlan& p, const double* x, int64_t N, cudaStream_t s);
// Jacobi eigensolve of every Gram (FP64), singular values, and the
// shrinkage matrix for thresholds beta[g*Q+q] * weights0[(g*Q+q)*lg + i].
// weights0/beta may be null (no thresholding: M = I - I = 0... only sigma used).
// rel_floor: eigenvalues <= rel_floor * lambda_max count as 0 (the rounding
// floor of the Gram; 0 keeps every nonnegative eigenvalue).
void nuc_eig(const NucPlan& p, const double* weights0, const double* beta, double* nuc_values, cudaStream_t s,
             double rel_floor = 0.0);
// v0 <- Z M (rows of Z = pixels).
void nuc_reconstruct(const NucPlan& p, const float* xhat, float* v0, cudaStream_t s);

// Window values of one facet along one axis (restated triangular apodisation).
std::vector<double> window_1d(int q, const std::vector<int>& base_start, const std::vector<int>& over_start,
                              const std::vector<int>& end, int window);

}  // namespace fhs
