// Host side of the device Broyden density mixer (src/mixers/broyden.hpp:26-160): the
// ring of difference vectors and the small linear solve of broyden_extrapolation.
// The vectors stay on the device; the host sees only their dot products.
//
// One call of the mixer (operator(), broyden.hpp:107-160) with input vin and output
// vout, ff = vout - vin:
//   * from the second call on, slot pos = (last + 1) % max_size of the ring takes
//     df = ff - f_old and dv = vin - vin_old, both divided by max(1e-8, |df|);
//   * f_old = ff, vin_old = vin;
//   * with n = min(calls - 1, max_size) slots in use:
//     vin += mix ff - sum_i c_i (mix df_i + dv_i), where c = ww^2 x and
//     beta x = work, with beta_ij = ww^2 df_i . df_j off the diagonal,
//     beta_ii = w0^2 + ww^2, work_i = df_i . ff, w0 = 0.01, ww = 5.
// The reference solves beta x = work with LAPACK dgelsd (least_squares.hpp:27-54).
// beta = ww^2 G + w0^2 I plus a non-negative diagonal, with G the Gram matrix of the df
// (each of norm at most 1), so it is symmetric positive definite with every eigenvalue
// at least w0^2.  Its least-squares solution is then the unique solution, which a
// Cholesky factorisation gives.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

namespace inqb {

struct BroydenRing {
  int max_size = 4;
  double mix = 0.3;
  int calls = 0, last = -1;

  // Starts one mixer call: the ring slot that takes this call's differences, or -1 on
  // the first call.
  int begin() {
    ++calls;
    return calls > 1 ? (last + 1) % max_size : -1;
  }
  void filled(int pos) {
    if (pos >= 0) last = pos;
  }
  int used() const { return std::min(calls - 1, max_size); }
};

// Solves a x = b in place (b becomes x) for a symmetric positive-definite n x n matrix
// a (row-major, overwritten by its Cholesky factor).  Returns false if a pivot is not
// positive.
inline bool spd_solve(int n, std::vector<double>& a, std::vector<double>& b) {
  for (int j = 0; j < n; j++) {
    double d = a[(size_t)j * n + j];
    for (int k = 0; k < j; k++) d -= a[(size_t)j * n + k] * a[(size_t)j * n + k];
    if (!(d > 0.0)) return false;
    const double l = std::sqrt(d);
    a[(size_t)j * n + j] = l;
    for (int i = j + 1; i < n; i++) {
      double s = a[(size_t)i * n + j];
      for (int k = 0; k < j; k++) s -= a[(size_t)i * n + k] * a[(size_t)j * n + k];
      a[(size_t)i * n + j] = s / l;
    }
  }
  for (int i = 0; i < n; i++) {  // L y = b
    double s = b[i];
    for (int k = 0; k < i; k++) s -= a[(size_t)i * n + k] * b[k];
    b[i] = s / a[(size_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {  // L^T x = y
    double s = b[i];
    for (int k = i + 1; k < n; k++) s -= a[(size_t)k * n + i] * b[k];
    b[i] = s / a[(size_t)i * n + i];
  }
  return true;
}

// The order of the dot products broyden_coefficients reads for n slots in use: first
// df_i . df_j for i < j < n (row by row), then df_i . ff for i < n.
inline int broyden_num_dots(int n) { return n * (n - 1) / 2 + n; }

// c [n] = ww^2 x for broyden_extrapolation from the dot products in the order above.
// Returns false if the system is not positive definite (a non-finite dot product).
inline bool broyden_coefficients(int n, const double* dots, double* c) {
  const double w0 = 0.01, ww = 5.0;
  std::vector<double> beta((size_t)n * n), work(n);
  int k = 0;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++, k++) beta[(size_t)i * n + j] = beta[(size_t)j * n + i] = ww * ww * dots[k];
  for (int i = 0; i < n; i++) beta[(size_t)i * n + i] = w0 * w0 + ww * ww;
  for (int i = 0; i < n; i++) work[i] = dots[k + i];
  if (!spd_solve(n, beta, work)) return false;
  for (int i = 0; i < n; i++) {
    if (!std::isfinite(work[i])) return false;
    c[i] = ww * ww * work[i];
  }
  return true;
}

}  // namespace inqb
