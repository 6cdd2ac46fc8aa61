// Host set-up of a B-spline interpolation axis (knots, band LU, reciprocal spans).
#pragma once

#include <vector>

namespace cfd2lcs {

template <typename R>
struct SplineAxisHost {
  int n = 0, k = 0;
  std::vector<R> t;     // n + k knots
  std::vector<R> lu;    // (2k-1) x n band LU, column-major, diagonal in row k (1-based)
  std::vector<R> rinv;  // 6 reciprocal knot spans per interval
  std::vector<R> tu;    // per interval l, pair at 2(l-1): t(l), and 1/h where the knots the basis
                        // depends on are equally spaced by h (else 0)
  // x: strictly increasing abscissae (the padded coordinate line); order k.
  bool build(const std::vector<R> &x, int order);
};

// Band LU of one axis in the pull form the device sweeps read, 8 values per row r (0-based):
// [j-1] the factor of L multiplying y(r-j) in the forward sweep, [3+j-1] the factor of U
// multiplying x(r+j) in the backward sweep (j = 1 .. k-1), [6] 1 / U(r,r).
template <typename R>
std::vector<R> spline_pull_table(const SplineAxisHost<R> &A) {
  const int n = A.n, k = A.k, nr = 2 * k - 1, mid = k;
  auto W = [&](int r, int c) { return A.lu[(size_t)(r - 1) + (size_t)nr * (c - 1)]; };
  std::vector<R> p((size_t)8 * n, R(0));
  for (int i = 1; i <= n; i++) {
    for (int j = 1; j <= k - 1; j++) {
      if (i - j >= 1) p[(size_t)8 * (i - 1) + j - 1] = W(mid + j, i - j);
      if (i + j <= n) p[(size_t)8 * (i - 1) + 3 + j - 1] = W(mid - j, i + j);
    }
    p[(size_t)8 * (i - 1) + 6] = R(1) / W(mid, i);
  }
  return p;
}

// The same factors arranged for the transposed solve (L U)^T f = c, used by the adjoint of a fit:
// U^T z = c forward, z(r) = (c(r) - sum_j U(r-j,r) z(r-j)) / U(r,r), with U(r-j,r) at [j-1] and
// 1/U(r,r) at [6]; then L^T f = z backward, f(r) = z(r) - sum_j L(r+j,r) f(r+j), with L(r+j,r)
// at [3+j-1].
template <typename R>
std::vector<R> spline_pull_table_transposed(const std::vector<R> &p, int n) {
  std::vector<R> t((size_t)8 * n, R(0));
  for (int r = 0; r < n; r++) {
    for (int j = 1; j <= 3; j++) {
      if (r - j >= 0) t[(size_t)8 * r + j - 1] = p[(size_t)8 * (r - j) + 3 + j - 1];
      if (r + j < n) t[(size_t)8 * r + 3 + j - 1] = p[(size_t)8 * (r + j) + j - 1];
    }
    t[(size_t)8 * r + 6] = p[(size_t)8 * r + 6];
  }
  return t;
}

}  // namespace cfd2lcs
