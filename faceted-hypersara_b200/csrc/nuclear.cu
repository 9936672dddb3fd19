// Faceted nuclear-norm prox on B200 (sm_100a).
//
// Replaces the per-facet SVD prox of src/fhs/fhs_update_dual_lowrankness.m:40-45
// (and src/hs/hs_update_dual_lowrankness_serial.m:37-42 with one facet and no
// window):  Z = v0 + D .* xhat_q (pixels x L), Z = U S V^T,
// v0 <- Z - U diag(max(S - beta w0, 0)) V^T.
// Since Z V = U S, the update equals v0 <- Z (I - V diag(shrink) V^T) with
// shrink_i = max(s_i - beta w0_i, 0) / s_i: the only dense contraction is the
// L x L Gram Z^T Z (split over pixel chunks, FP32 products, FP64 sums), then
// an FP64 Jacobi eigensolve per facet gives V and s_i = sqrt(lambda_i), and
// the rank-L update is one streaming pass over Z.
#include "nuclear.cuh"
#include "tf32.cuh"

#include <algorithm>
#include <cmath>

namespace fhs {

namespace {

constexpr int kSub = 64;  // pixels staged per Gram step

template <int MAXL>
__device__ __forceinline__ void load_z_row(const NucFacet& f, int g, int lg, int Ny, int64_t npix, int64_t p,
                                           const float* __restrict__ xhat, const float* __restrict__ v0,
                                           const float* __restrict__ wy, const float* __restrict__ wx,
                                           int64_t v0_group, int64_t P, float z[MAXL]) {
  const int ny = f.y1 - f.y0;
  const int lx = (int)(p / ny), ly = (int)(p - (int64_t)lx * ny);
  const float w = wy[f.wy_off + ly] * wx[f.wx_off + lx];
  const int64_t pix = (int64_t)(f.x0 + lx) * Ny + (f.y0 + ly);
#pragma unroll
  for (int l = 0; l < MAXL; ++l) {
    if (l < lg) {
      float v = w * xhat[((int64_t)g * lg + l) * npix + pix];
      if (v0) v += v0[(int64_t)g * v0_group + f.v0_off + (int64_t)l * P + p];
      z[l] = v;
    }
  }
}

template <int MAXL>
__global__ void __launch_bounds__(256) gram_kernel(const NucFacet* __restrict__ facets, int Q, int lg, int Ny,
                                                   int64_t npix, const float* __restrict__ xhat,
                                                   const float* __restrict__ v0, const float* __restrict__ wy,
                                                   const float* __restrict__ wx, int64_t v0_group,
                                                   int max_chunks, float* __restrict__ part) {
  constexpr int E = (MAXL * MAXL + 255) / 256;
  __shared__ float Z[kSub][MAXL + 1];
  const int chunk = blockIdx.x, q = blockIdx.y, g = blockIdx.z;
  const NucFacet f = facets[q];
  if (chunk >= f.nchunks) return;
  const int64_t P = (int64_t)(f.y1 - f.y0) * (f.x1 - f.x0);
  const int64_t c0 = (int64_t)chunk * kNucChunk, c1 = min(P, c0 + kNucChunk);
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  for (int64_t base = c0; base < c1; base += kSub) {
    // stage kSub rows of Z
    for (int idx = threadIdx.x; idx < kSub; idx += blockDim.x) {
      const int64_t p = base + idx;
      float z[MAXL];
      if (p < c1) {
        load_z_row<MAXL>(f, g, lg, Ny, npix, p, xhat, v0, wy, wx, v0_group, P, z);
      } else {
#pragma unroll
        for (int l = 0; l < MAXL; ++l) z[l] = 0.f;
      }
#pragma unroll
      for (int l = 0; l < MAXL; ++l)
        if (l < lg) Z[idx][l] = z[l];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ent = threadIdx.x + 256 * e;
      if (ent < lg * lg) {
        const int i = ent / lg, j = ent - i * lg;
        float a = acc[e];
        for (int r = 0; r < kSub; ++r) a = fmaf(Z[r][i], Z[r][j], a);
        acc[e] = a;
      }
    }
    __syncthreads();
  }
  float* out = part + (((int64_t)g * Q + q) * max_chunks + chunk) * lg * lg;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int ent = threadIdx.x + 256 * e;
    if (ent < lg * lg) out[ent] = acc[e];
  }
}

// Gram of up to 16 channels on the tensor cores.  A stage of kGStage pixels
// of Z is staged channel-major (pitch kGPitch = 4 mod 32: the fragment reads
// of a warp hit 32 distinct banks); warp w contracts pixels [32 w, 32 w + 32)
// of the stage: with A = Z^T (16 channels x 8 pixels) the B fragments of the
// two 8-channel column blocks are A's own elements, so one k-step is four
// shared loads, one split and 2 x 3 MMAs.  Each stage's products start from
// zero in the tensor core and are added to the running FP32 sums, so the
// in-core accumulation never spans more than 32 pixels.
constexpr int kGStage = 256;
constexpr int kGPitch = kGStage + 4;

__global__ void __launch_bounds__(256) gram_mma_kernel(const NucFacet* __restrict__ facets, int Q, int lg, int Ny,
                                                       int64_t npix, const float* __restrict__ xhat,
                                                       const float* __restrict__ v0, const float* __restrict__ wy,
                                                       const float* __restrict__ wx, int64_t v0_group,
                                                       int max_chunks, float* __restrict__ part) {
  __shared__ float Zs[16 * kGPitch];
  __shared__ float red[8][256];
  const int chunk = blockIdx.x, q = blockIdx.y, g = blockIdx.z;
  const NucFacet f = facets[q];
  if (chunk >= f.nchunks) return;
  const int64_t P = (int64_t)(f.y1 - f.y0) * (f.x1 - f.x0);
  const int64_t c0 = (int64_t)chunk * kNucChunk, c1 = min(P, c0 + kNucChunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gr = lane >> 2, t = lane & 3;
  float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  for (int64_t base = c0; base < c1; base += kGStage) {
    {
      const int64_t p = base + threadIdx.x;
      float z[16];
      if (p < c1) {
        load_z_row<16>(f, g, lg, Ny, npix, p, xhat, v0, wy, wx, v0_group, P, z);
      } else {
#pragma unroll
        for (int l = 0; l < 16; ++l) z[l] = 0.f;
      }
#pragma unroll
      for (int l = 0; l < 16; ++l) Zs[l * kGPitch + threadIdx.x] = l < lg ? z[l] : 0.f;
    }
    __syncthreads();
    float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int k0 = warp * 32 + ks * 8;
      const float a0 = Zs[gr * kGPitch + k0 + t], a1 = Zs[(gr + 8) * kGPitch + k0 + t];
      const float a2 = Zs[gr * kGPitch + k0 + t + 4], a3 = Zs[(gr + 8) * kGPitch + k0 + t + 4];
      const FragA3 A = frag_a3(a0, a1, a2, a3);
      mma3xtf32(d[0], A, frag_b3(a0, a2));  // channels 0-7
      mma3xtf32(d[1], A, frag_b3(a1, a3));  // channels 8-15
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[nt][k] += d[nt][k];
    __syncthreads();
  }
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    red[warp][gr * 16 + 8 * nt + 2 * t] = acc[nt][0];
    red[warp][gr * 16 + 8 * nt + 2 * t + 1] = acc[nt][1];
    red[warp][(gr + 8) * 16 + 8 * nt + 2 * t] = acc[nt][2];
    red[warp][(gr + 8) * 16 + 8 * nt + 2 * t + 1] = acc[nt][3];
  }
  __syncthreads();
  const int i = threadIdx.x >> 4, j = threadIdx.x & 15;
  if (i < lg && j < lg) {
    float v = 0.f;
#pragma unroll
    for (int w = 0; w < 8; ++w) v += red[w][threadIdx.x];
    part[(((int64_t)g * Q + q) * max_chunks + chunk) * lg * lg + i * lg + j] = v;
  }
}

__global__ void gram_reduce_kernel(const NucFacet* __restrict__ facets, int Q, int lg, int max_chunks,
                                   const float* __restrict__ part, double* __restrict__ gram) {
  const int q = blockIdx.x, g = blockIdx.y;
  const int nch = facets[q].nchunks;
  const float* src = part + ((int64_t)g * Q + q) * max_chunks * lg * lg;
  for (int ent = threadIdx.x; ent < lg * lg; ent += blockDim.x) {
    double a = 0.0;
    for (int c = 0; c < nch; ++c) a += (double)src[(int64_t)c * lg * lg + ent];
    gram[((int64_t)g * Q + q) * lg * lg + ent] = a;
  }
}

// Parallel-ordered cyclic Jacobi (round-robin pairing) on one symmetric
// lg x lg matrix per CTA, FP64, at most kMaxSweeps sweeps.
constexpr int kMaxSweeps = 40;

__device__ __forceinline__ int rr_elem(int i, int r, int m) { return i == 0 ? 0 : ((r + i - 1) % (m - 1)) + 1; }

__global__ void __launch_bounds__(256) eig_kernel(const double* __restrict__ gram, int lg,
                                                  const double* __restrict__ weights0,
                                                  const double* __restrict__ beta, float* __restrict__ Mout,
                                                  double* __restrict__ sigma_out, double* __restrict__ nuc_values,
                                                  double rel_floor) {
  extern __shared__ double sh[];
  const int n = lg;
  double* A = sh;            // n*n
  double* V = A + n * n;     // n*n
  __shared__ double cs_c[kNucMaxL / 2 + 1], cs_s[kNucMaxL / 2 + 1];
  __shared__ double red[256];
  __shared__ double sig[kNucMaxL], shr[kNucMaxL];
  __shared__ int perm[kNucMaxL];
  __shared__ int done;
  const int id = blockIdx.x;  // g*Q + q
  const double* G = gram + (int64_t)id * n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    A[e] = 0.5 * (G[i * n + j] + G[j * n + i]);
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int m = n + (n & 1);
  for (int sweep = 0; sweep < kMaxSweeps && n > 1; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e - i * n;
      if (i == j)
        dg += A[e] * A[e];
      else
        off += A[e] * A[e];
    }
    red[threadIdx.x] = off;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
      if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
      __syncthreads();
    }
    const double offs = red[0];
    __syncthreads();
    red[threadIdx.x] = dg;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
      if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
      __syncthreads();
    }
    if (threadIdx.x == 0) done = (offs <= 1e-30 * red[0]) || offs == 0.0;
    __syncthreads();
    if (done) break;
    for (int r = 0; r < m - 1; ++r) {
      if (threadIdx.x < m / 2) {
        const int k = threadIdx.x;
        const int p = rr_elem(k, r, m), q = rr_elem(m - 1 - k, r, m);
        double c = 1.0, s = 0.0;
        if (p < n && q < n) {
          const double apq = A[p * n + q];
          if (fabs(apq) > 1e-300) {
            const double tau = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
            const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs_c[k] = c;
        cs_s[k] = s;
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < (m / 2) * n; idx += blockDim.x) {
        const int k = idx / n, col = idx - k * n;
        const int p = rr_elem(k, r, m), q = rr_elem(m - 1 - k, r, m);
        if (p < n && q < n) {
          const double c = cs_c[k], s = cs_s[k];
          const double ap = A[p * n + col], aq = A[q * n + col];
          A[p * n + col] = c * ap - s * aq;
          A[q * n + col] = s * ap + c * aq;
        }
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < (m / 2) * n; idx += blockDim.x) {
        const int k = idx / n, row = idx - k * n;
        const int p = rr_elem(k, r, m), q = rr_elem(m - 1 - k, r, m);
        if (p < n && q < n) {
          const double c = cs_c[k], s = cs_s[k];
          const double ap = A[row * n + p], aq = A[row * n + q];
          A[row * n + p] = c * ap - s * aq;
          A[row * n + q] = s * ap + c * aq;
          const double vp = V[row * n + p], vq = V[row * n + q];
          V[row * n + p] = c * vp - s * vq;
          V[row * n + q] = s * vp + c * vq;
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = 0; i < n; ++i) {  // selection sort, descending eigenvalues
      int b = i;
      for (int j = i + 1; j < n; ++j)
        if (A[perm[j] * n + perm[j]] > A[perm[b] * n + perm[b]]) b = j;
      const int t = perm[i];
      perm[i] = perm[b];
      perm[b] = t;
    }
    double tot = 0.0;
    // eigenvalues under the Gram's rounding floor are indistinguishable from 0
    const double floor_lam = rel_floor * fmax(A[perm[0] * n + perm[0]], 0.0);
    for (int i = 0; i < n; ++i) {
      const double lam = A[perm[i] * n + perm[i]];
      const double sv = lam > floor_lam ? sqrt(lam) : 0.0;
      sig[i] = sv;
      tot += sv;
      double th = 0.0;
      if (beta && weights0) th = beta[id] * weights0[(int64_t)id * n + i];
      shr[i] = sv > 0.0 ? fmax(sv - th, 0.0) / sv : 0.0;
      if (sigma_out) sigma_out[(int64_t)id * n + i] = sv;
    }
    if (nuc_values) nuc_values[id] = tot;
  }
  __syncthreads();
  if (Mout) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int a = e / n, b = e - a * n;
      double acc = (a == b) ? 1.0 : 0.0;
      for (int i = 0; i < n; ++i) acc -= V[a * n + perm[i]] * shr[i] * V[b * n + perm[i]];
      Mout[(int64_t)id * n * n + e] = (float)acc;
    }
  }
}

template <int MAXL>
__global__ void __launch_bounds__(256) reconstruct_kernel(const NucFacet* __restrict__ facets, int Q, int lg,
                                                          int Ny, int64_t npix, const float* __restrict__ xhat,
                                                          float* __restrict__ v0, const float* __restrict__ wy,
                                                          const float* __restrict__ wx, int64_t v0_group,
                                                          const float* __restrict__ Mall) {
  __shared__ float M[MAXL * MAXL];
  const int chunk = blockIdx.x, q = blockIdx.y, g = blockIdx.z;
  const NucFacet f = facets[q];
  if (chunk >= f.nchunks) return;
  const float* Mg = Mall + ((int64_t)g * Q + q) * lg * lg;
  for (int e = threadIdx.x; e < lg * lg; e += blockDim.x) M[e] = Mg[e];
  __syncthreads();
  const int64_t P = (int64_t)(f.y1 - f.y0) * (f.x1 - f.x0);
  const int64_t c0 = (int64_t)chunk * kNucChunk, c1 = min(P, c0 + kNucChunk);
  for (int64_t p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
    float z[MAXL];
    load_z_row<MAXL>(f, g, lg, Ny, npix, p, xhat, v0, wy, wx, v0_group, P, z);
    float* dst = v0 + (int64_t)g * v0_group + f.v0_off + p;
    for (int b = 0; b < lg; ++b) {
      float acc = 0.f;
#pragma unroll
      for (int a = 0; a < MAXL; ++a)
        if (a < lg) acc = fmaf(z[a], M[a * lg + b], acc);
      dst[(int64_t)b * P] = acc;
    }
  }
}

}  // namespace

std::vector<double> window_1d(int q, const std::vector<int>& base_start, const std::vector<int>& over_start,
                              const std::vector<int>& end, int window) {
  const int n = end[q] - over_start[q];
  std::vector<double> w(n, 1.0);
  if (window == FHS_WINDOW_NONE) return w;
  const int ol = base_start[q] - over_start[q];
  for (int i = 0; i < ol; ++i) w[i] = (i + 1.0) / (ol + 1.0);
  if (q + 1 < (int)base_start.size()) {
    const int orr = base_start[q + 1] - over_start[q + 1];
    for (int i = 0; i < orr; ++i) w[n - orr + i] *= 1.0 - (i + 1.0) / (orr + 1.0);
  }
  return w;
}

void nuc_plan_init(NucPlan& p, int Ny, int Nx, int Qy, int Qx, const std::vector<int>& sy,
                   const std::vector<int>& sx, int oy, int ox, int window, int n_groups, int lg, cudaStream_t s) {
  FHS_CHECK(lg >= 1 && lg <= kNucMaxL, FHS_ERR_UNSUPPORTED, "channels per group must be in [1, 64]");
  FHS_CHECK((int)sy.size() == Qy + 1 && (int)sx.size() == Qx + 1, FHS_ERR_INVALID_ARG, "bad facet splits");
  p.Ny = Ny;
  p.Nx = Nx;
  p.Qy = Qy;
  p.Qx = Qx;
  p.Q = Qy * Qx;
  p.n_groups = n_groups;
  p.lg = lg;
  auto axis = [&](const std::vector<int>& sp, int Q, int ov, int N, std::vector<int>& bs, std::vector<int>& os,
                  std::vector<int>& en) {
    FHS_CHECK(sp[0] == 0 && sp[Q] == N, FHS_ERR_INVALID_ARG, "facet splits must start at 0 and end at N");
    for (int q = 0; q < Q; ++q) {
      FHS_CHECK(sp[q + 1] > sp[q], FHS_ERR_INVALID_ARG, "empty facet");
      bs.push_back(sp[q]);
      os.push_back(q > 0 ? std::max(sp[q] - ov, 0) : sp[q]);
      en.push_back(sp[q + 1]);
    }
    for (int q = 0; q + 1 < Q; ++q)
      FHS_CHECK(os[q + 1] >= bs[q], FHS_ERR_UNSUPPORTED, "facet overlap larger than a facet");
  };
  std::vector<int> bsy, osy, eny, bsx, osx, enx;
  axis(sy, Qy, oy, Ny, bsy, osy, eny);
  axis(sx, Qx, ox, Nx, bsx, osx, enx);
  std::vector<float> hwy, hwx;
  std::vector<int64_t> wyo(Qy), wxo(Qx);
  for (int q = 0; q < Qy; ++q) {
    wyo[q] = hwy.size();
    for (double v : window_1d(q, bsy, osy, eny, window)) hwy.push_back((float)v);
  }
  for (int q = 0; q < Qx; ++q) {
    wxo[q] = hwx.size();
    for (double v : window_1d(q, bsx, osx, enx, window)) hwx.push_back((float)v);
  }
  p.facets.clear();
  int64_t off = 0;
  p.max_chunks = 0;
  for (int qx = 0; qx < Qx; ++qx)
    for (int qy = 0; qy < Qy; ++qy) {
      NucFacet f;
      f.y0 = osy[qy];
      f.y1 = eny[qy];
      f.x0 = osx[qx];
      f.x1 = enx[qx];
      f.v0_off = off;
      f.wy_off = wyo[qy];
      f.wx_off = wxo[qx];
      const int64_t P = (int64_t)(f.y1 - f.y0) * (f.x1 - f.x0);
      f.nchunks = ceil_div(P, kNucChunk);
      p.max_chunks = std::max(p.max_chunks, f.nchunks);
      off += P * lg;
      p.facets.push_back(f);
    }
  p.v0_group = off;
  // cover lists: which facets (along each axis) contain a pixel row/column
  auto cover = [&](int N, int Q, const std::vector<int>& os, const std::vector<int>& en) {
    std::vector<int> c((size_t)N * 2, -1);
    for (int q = 0; q < Q; ++q)
      for (int i = os[q]; i < en[q]; ++i) {
        if (c[2 * i] < 0)
          c[2 * i] = q;
        else
          c[2 * i + 1] = q;
      }
    return c;
  };
  const auto cy = cover(Ny, Qy, osy, eny), cx = cover(Nx, Qx, osx, enx);
  p.d_facets.alloc(p.facets.size());
  p.d_facets.upload(p.facets.data(), p.facets.size(), s);
  p.wy.alloc(hwy.size());
  p.wy.upload(hwy.data(), hwy.size(), s);
  p.wx.alloc(hwx.size());
  p.wx.upload(hwx.data(), hwx.size(), s);
  p.cover_y.alloc(cy.size());
  p.cover_y.upload(cy.data(), cy.size(), s);
  p.cover_x.alloc(cx.size());
  p.cover_x.upload(cx.data(), cx.size(), s);
  p.gram_part.alloc((size_t)n_groups * p.Q * p.max_chunks * lg * lg);
  p.gram.alloc((size_t)n_groups * p.Q * lg * lg);
  p.shrinkM.alloc((size_t)n_groups * p.Q * lg * lg);
  p.sigma.alloc((size_t)n_groups * p.Q * lg);
  FHS_CUDA(cudaStreamSynchronize(s));
}

#define FHS_NUC_DISPATCH(KERNEL, GRID, ...)                                   \
  do {                                                                        \
    if (p.lg <= 8)                                                            \
      KERNEL<8><<<GRID, 256, 0, s>>>(__VA_ARGS__);                            \
    else if (p.lg <= 16)                                                      \
      KERNEL<16><<<GRID, 256, 0, s>>>(__VA_ARGS__);                           \
    else if (p.lg <= 32)                                                      \
      KERNEL<32><<<GRID, 256, 0, s>>>(__VA_ARGS__);                           \
    else                                                                      \
      KERNEL<64><<<GRID, 256, 0, s>>>(__VA_ARGS__);                           \
  } while (0)

void nuc_gram(const NucPlan& p, const float* xhat, const float* v0, cudaStream_t s) {
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  dim3 grid(p.max_chunks, p.Q, p.n_groups);
  if (p.lg <= 16)  // tensor cores (3xTF32)
    gram_mma_kernel<<<grid, 256, 0, s>>>(p.d_facets.p, p.Q, p.lg, p.Ny, npix, xhat, v0, p.wy.p, p.wx.p, p.v0_group,
                                         p.max_chunks, p.gram_part.p);
  else
    FHS_NUC_DISPATCH(gram_kernel, grid, p.d_facets.p, p.Q, p.lg, p.Ny, npix, xhat, v0, p.wy.p, p.wx.p, p.v0_group,
                     p.max_chunks, p.gram_part.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  gram_reduce_kernel<<<dim3(p.Q, p.n_groups), 256, 0, s>>>(p.d_facets.p, p.Q, p.lg, p.max_chunks, p.gram_part.p,
                                                            p.gram.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

// ------------------------------------------------------------ FP64 Gram
// G = X^T X of an FP64 [L][N] matrix (channel planes), for nuclear_norm:
// singular values from a Gram eigensolve lose sqrt(Gram error) x sigma_max
// of absolute accuracy, so a nearly low-rank cube needs the Gram in FP64.
// CTA = a pixel range staged 64 pixels at a time; thread (bi, bj) owns the
// 4 x 4 block of channel pairs (4 bi.., 4 bj..), bi <= bj; per-CTA partials
// are summed in a fixed order (deterministic).
namespace {
constexpr int kG64Pix = 64;
constexpr int kG64PerCta = 16384;

__global__ void __launch_bounds__(256) gram64_partial_kernel(const double* __restrict__ x, int64_t N, int L,
                                                             double* __restrict__ part) {
  __shared__ double sx[kG64Pix][kNucMaxL + 1];
  const int nb = (L + 3) / 4;
  const int bi = threadIdx.x / 16, bj = threadIdx.x % 16;
  const bool active = bi < nb && bj < nb && bi <= bj;
  for (int idx = threadIdx.x; idx < kG64Pix * (kNucMaxL + 1); idx += blockDim.x) (&sx[0][0])[idx] = 0.0;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
  const int64_t p0 = (int64_t)blockIdx.x * kG64PerCta;
  const int64_t p1 = min(N, p0 + kG64PerCta);
  for (int64_t base = p0; base < p1; base += kG64Pix) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kG64Pix * L; idx += blockDim.x) {
      const int l = idx / kG64Pix, q = idx - l * kG64Pix;
      const int64_t pix = base + q;
      sx[q][l] = pix < p1 ? x[(int64_t)l * N + pix] : 0.0;
    }
    __syncthreads();
    if (active) {
      for (int q = 0; q < kG64Pix; ++q) {
        double a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          a[r] = sx[q][4 * bi + r];
          b[r] = sx[q][4 * bj + r];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
      }
    }
  }
  if (active) {
    double* o = part + (size_t)blockIdx.x * kNucMaxL * kNucMaxL;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int i = 4 * bi + r, j = 4 * bj + c;
        if (i < L && j < L) o[i * kNucMaxL + j] = acc[r][c];
      }
  }
}

__global__ void gram64_reduce_kernel(const double* __restrict__ part, int nparts, int L, double* __restrict__ gram) {
  const int i = blockIdx.x, j = threadIdx.x;
  if (j >= L) return;
  const int a = min(i, j), b = max(i, j);  // partials hold the upper triangle
  double t = 0.0;
  for (int k = 0; k < nparts; ++k) t += part[(size_t)k * kNucMaxL * kNucMaxL + a * kNucMaxL + b];
  gram[i * L + j] = t;
}
}  // namespace

void nuc_gram_fp64(const NucPlan& p, const double* x, int64_t N, cudaStream_t s) {
  FHS_CHECK(p.n_groups == 1 && p.Q == 1, FHS_ERR_INVALID_ARG, "FP64 Gram: one group, one facet");
  const int nparts = (int)((N + kG64PerCta - 1) / kG64PerCta);
  DevBuf<double> part;
  part.alloc((size_t)nparts * kNucMaxL * kNucMaxL);
  gram64_partial_kernel<<<nparts, 256, 0, s>>>(x, N, p.lg, part.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  gram64_reduce_kernel<<<p.lg, 64, 0, s>>>(part.p, nparts, p.lg, p.gram.p);
  count_launch();
  FHS_LAUNCH_CHECK();
  FHS_CUDA(cudaStreamSynchronize(s));  // part is released on return
}

void nuc_eig(const NucPlan& p, const double* weights0, const double* beta, double* nuc_values, cudaStream_t s,
             double rel_floor) {
  const size_t smem = 2 * (size_t)p.lg * p.lg * sizeof(double);
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev < 64 && !attr_set[dev]) {
    FHS_CUDA(cudaFuncSetAttribute(eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 64 * 64 * 8));
    attr_set[dev] = true;
  }
  eig_kernel<<<p.n_groups * p.Q, 256, smem, s>>>(p.gram.p, p.lg, weights0, beta, p.shrinkM.p, p.sigma.p,
                                                  nuc_values, rel_floor);
  count_launch();
  FHS_LAUNCH_CHECK();
}

void nuc_reconstruct(const NucPlan& p, const float* xhat, float* v0, cudaStream_t s) {
  const int64_t npix = (int64_t)p.Ny * p.Nx;
  dim3 grid(p.max_chunks, p.Q, p.n_groups);
  FHS_NUC_DISPATCH(reconstruct_kernel, grid, p.d_facets.p, p.Q, p.lg, p.Ny, npix, xhat, v0, p.wy.p, p.wx.p,
                   p.v0_group, p.shrinkM.p);
  count_launch();
  FHS_LAUNCH_CHECK();
}

}  // namespace fhs
