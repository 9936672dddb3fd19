// Host-side FP64 min-max NUFFT interpolator tables (see minmax.cpp).
#pragma once

#include <vector>

namespace fhs {

struct MinMaxAxis {
  int N = 0, K = 0, J = 0, n_samples = 0;
  std::vector<double> cos_coefs;  // scaling cosine series a_0..a_L
  std::vector<double> scale;      // s_n, n = 0..N-1
  std::vector<double> table_re;   // h_j(dk) real part, [J][n_samples+1]
  std::vector<double> table_im;   // imaginary part
  // degree kPolyDegree least-squares polynomials of every tap in
  // s = (dk - J/2) - 1/2 in [-1/2, 1/2): poly[(j*2 + part)*(kPolyDegree+1) + k]
  std::vector<double> poly;
  // the same taps without their phase: h_j(dk) = exp(i pi (dk - j)/K) c_j(dk)
  // with c_j real; degree kPolyDegree fits poly_real[j*(kPolyDegree+1) + k]
  std::vector<double> poly_real;
};

constexpr int kPolyDegree = 8;

// Tables for one axis: N image pixels, K grid cells, J taps.
MinMaxAxis build_minmax_axis(int N, int K, int J, int n_samples, int n_cos = 6);

}  // namespace fhs
