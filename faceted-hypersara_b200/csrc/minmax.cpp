// Host-side FP64 construction of the min-max NUFFT interpolator.
//
// Restates Fessler & Sutton 2003 (the method of op_p_nufft in the
// RI-measurement-operator submodule, called at
// lib/operators/util_gen_measurement_operator_synth.m:86 with 'minmax:kb'):
// for J neighbours k0+1..k0+J of om (k0 = floor(om/gamma - J/2)), the
// coefficients minimising the worst-case interpolation error are
// g = (A^H A)^{-1} A^H b with A[n,j] = s_n exp(-i gamma (k0+j) n),
// b_n = exp(-i om (n - N/2)).  The scaling s_n is a cosine series fitted to
// the reciprocal Fourier transform of the order-0 Kaiser-Bessel kernel
// (alpha = 2.34 J), so every sum over n is a Dirichlet kernel.
//
// With the image placed at (n - N/2) mod K before the FFT, the per-tap
// coefficient depends on the fractional offset dk = om/gamma - k0 only:
// h_j(dk) = exp(i pi (dk - j)/K) (R^{-1} r(dk))_j, R[j,l] = S2(gamma(j-l)),
// r_j = S(gamma(dk - j)).  This file tabulates h_j on a uniform grid of dk.
#include "minmax.h"

#include <cmath>
#include <stdexcept>
#include <vector>

namespace fhs {

namespace {

double bessel_i0(double x) {
  // power series sum (x/2)^{2k} / (k!)^2, converges for all x used here (< 20)
  double sum = 1.0, term = 1.0, q = 0.25 * x * x;
  for (int k = 1; k < 500; ++k) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  return sum;
}

double kb_ft(double nu, int J, double alpha) {
  const double z2 = alpha * alpha - (M_PI * J * nu) * (M_PI * J * nu);
  double v;
  if (z2 > 0) {
    const double z = std::sqrt(z2);
    v = z > 0 ? std::sinh(z) / z : 1.0;
  } else {
    const double z = std::sqrt(-z2);
    v = z > 0 ? std::sin(z) / z : 1.0;
  }
  return J / bessel_i0(alpha) * v;
}

// D(x) = sin(pi N x / K) / sin(pi x / K), D(0) = N.
double dirichlet(double x, int N, int K) {
  const double den = std::sin(M_PI * x / K);
  if (std::fabs(den) < 1e-300) return (double)N;
  return std::sin(M_PI * N * x / K) / den;
}

// Householder least squares min ||B a - t|| (B: m x n, column-major).
std::vector<double> lstsq(std::vector<double> B, std::vector<double> t, int m, int n) {
  for (int k = 0; k < n; ++k) {
    double nrm = 0;
    for (int i = k; i < m; ++i) nrm += B[i + (size_t)m * k] * B[i + (size_t)m * k];
    nrm = std::sqrt(nrm);
    if (nrm == 0) throw std::runtime_error("rank-deficient scaling fit");
    const double alpha = B[k + (size_t)m * k] > 0 ? -nrm : nrm;
    std::vector<double> v(m, 0.0);
    for (int i = k; i < m; ++i) v[i] = B[i + (size_t)m * k];
    v[k] -= alpha;
    double vn = 0;
    for (int i = k; i < m; ++i) vn += v[i] * v[i];
    for (int j = k; j < n; ++j) {
      double d = 0;
      for (int i = k; i < m; ++i) d += v[i] * B[i + (size_t)m * j];
      const double f = 2.0 * d / vn;
      for (int i = k; i < m; ++i) B[i + (size_t)m * j] -= f * v[i];
    }
    double d = 0;
    for (int i = k; i < m; ++i) d += v[i] * t[i];
    const double f = 2.0 * d / vn;
    for (int i = k; i < m; ++i) t[i] -= f * v[i];
  }
  std::vector<double> a(n);
  for (int k = n - 1; k >= 0; --k) {
    double s = t[k];
    for (int j = k + 1; j < n; ++j) s -= B[k + (size_t)m * j] * a[j];
    a[k] = s / B[k + (size_t)m * k];
  }
  return a;
}

// Inverse of a small symmetric positive definite matrix (Gauss-Jordan, pivoting).
std::vector<double> invert(std::vector<double> A, int n) {
  std::vector<double> I(n * n, 0.0);
  for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (A[p * n + c] == 0) throw std::runtime_error("singular min-max matrix");
    if (p != c)
      for (int j = 0; j < n; ++j) {
        std::swap(A[p * n + j], A[c * n + j]);
        std::swap(I[p * n + j], I[c * n + j]);
      }
    const double d = A[c * n + c];
    for (int j = 0; j < n; ++j) {
      A[c * n + j] /= d;
      I[c * n + j] /= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = A[r * n + c];
      if (f == 0) continue;
      for (int j = 0; j < n; ++j) {
        A[r * n + j] -= f * A[c * n + j];
        I[r * n + j] -= f * I[c * n + j];
      }
    }
  }
  return I;
}

}  // namespace

MinMaxAxis build_minmax_axis(int N, int K, int J, int n_samples, int n_cos) {
  if (J < 2 || J > 8) throw std::runtime_error("J must be in [2, 8]");
  MinMaxAxis ax;
  ax.N = N;
  ax.K = K;
  ax.J = J;
  ax.n_samples = n_samples;
  const double alpha = 2.34 * J;
  const double c = (N - 1) / 2.0;
  // cosine-series fit of s_n = FT(0)/FT((n-c)/K)
  const int nb = n_cos + 1;
  std::vector<double> B((size_t)N * nb), t(N);
  const double ft0 = kb_ft(0.0, J, alpha);
  for (int n = 0; n < N; ++n) {
    t[n] = ft0 / kb_ft((n - c) / K, J, alpha);
    for (int l = 0; l < nb; ++l) B[n + (size_t)N * l] = std::cos(2.0 * M_PI * l * (n - c) / K);
  }
  ax.cos_coefs = lstsq(B, t, N, nb);
  ax.scale.resize(N);
  for (int n = 0; n < N; ++n) {
    double s = 0;
    for (int l = 0; l < nb; ++l) s += ax.cos_coefs[l] * std::cos(2.0 * M_PI * l * (n - c) / K);
    ax.scale[n] = s;
  }
  // two-sided alpha_l
  const int L = n_cos;
  std::vector<double> al(2 * L + 1, 0.0);
  al[L] = ax.cos_coefs[0];
  for (int l = 1; l <= L; ++l) al[L + l] = al[L - l] = ax.cos_coefs[l] / 2.0;
  // R[j,l] = sum_{l1,l2} al al D((j-l) - (l1+l2))
  std::vector<double> R(J * J, 0.0);
  for (int j = 0; j < J; ++j)
    for (int k = 0; k < J; ++k) {
      double acc = 0;
      for (int i1 = 0; i1 <= 2 * L; ++i1)
        for (int i2 = 0; i2 <= 2 * L; ++i2)
          acc += al[i1] * al[i2] * dirichlet((double)(j - k) - ((i1 - L) + (i2 - L)), N, K);
      R[j * J + k] = acc;
    }
  const std::vector<double> T = invert(R, J);
  // table h[j][t], dk = J/2 + t/n_samples
  ax.table_re.assign((size_t)J * (n_samples + 1), 0.0);
  ax.table_im.assign((size_t)J * (n_samples + 1), 0.0);
  std::vector<double> table_c((size_t)J * (n_samples + 1), 0.0);  // c_j(dk), real
  std::vector<double> r(J), cc(J);
  for (int ti = 0; ti <= n_samples; ++ti) {
    const double dk = J / 2.0 + (double)ti / n_samples;
    for (int j = 1; j <= J; ++j) {
      double acc = 0;
      for (int il = 0; il <= 2 * L; ++il) acc += al[il] * dirichlet(dk - j - (il - L), N, K);
      r[j - 1] = acc;
    }
    for (int j = 0; j < J; ++j) {
      double acc = 0;
      for (int k = 0; k < J; ++k) acc += T[j * J + k] * r[k];
      cc[j] = acc;
    }
    for (int j = 1; j <= J; ++j) {
      table_c[(size_t)(j - 1) * (n_samples + 1) + ti] = cc[j - 1];
      const double ph = M_PI / K * (dk - j);
      ax.table_re[(size_t)(j - 1) * (n_samples + 1) + ti] = std::cos(ph) * cc[j - 1];
      ax.table_im[(size_t)(j - 1) * (n_samples + 1) + ti] = std::sin(ph) * cc[j - 1];
    }
  }
  // polynomial fits of every tap (real and imaginary parts) over the table
  const int nt = kPolyDegree + 1, m = n_samples + 1;
  ax.poly.assign((size_t)J * 2 * nt, 0.0);
  std::vector<double> V((size_t)m * nt);
  for (int ti = 0; ti < m; ++ti) {
    const double sv = (double)ti / n_samples - 0.5;
    double pw = 1.0;
    for (int k = 0; k < nt; ++k) {
      V[ti + (size_t)m * k] = pw;
      pw *= sv;
    }
  }
  for (int j = 0; j < J; ++j)
    for (int part = 0; part < 2; ++part) {
      const std::vector<double>& tab = part ? ax.table_im : ax.table_re;
      std::vector<double> t(tab.begin() + (size_t)j * m, tab.begin() + (size_t)(j + 1) * m);
      const std::vector<double> c = lstsq(V, t, m, nt);
      for (int k = 0; k < nt; ++k) ax.poly[((size_t)j * 2 + part) * nt + k] = c[k];
    }
  ax.poly_real.assign((size_t)J * nt, 0.0);
  for (int j = 0; j < J; ++j) {
    std::vector<double> t(table_c.begin() + (size_t)j * m, table_c.begin() + (size_t)(j + 1) * m);
    const std::vector<double> c = lstsq(V, t, m, nt);
    for (int k = 0; k < nt; ++k) ax.poly_real[(size_t)j * nt + k] = c[k];
  }
  return ax;
}

}  // namespace fhs
