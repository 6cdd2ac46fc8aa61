// Host set-up of one spline axis: knots (dbknot, src/bspline/bspline_sub_module.f90:1737-1785),
// collocation matrix from the basis values at the abscissae and its band LU without
// pivoting (dbintk :1896-2036, dbnfac :2098-2184), plus reciprocal knot spans for the
// device basis evaluation.  Runs once per grid and order.
#include "spline_host.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace cfd2lcs {

template <typename R>
static void knots(const std::vector<R> &x, int n, int k, std::vector<R> &t) {
  t.assign(n + k, R(0));
  const R rnot = x[n - 1] + R(0.1) * (x[n - 1] - x[n - 2]);
  for (int j = 0; j < k; j++) {
    t[j] = x[0];
    t[n + j] = rnot;
  }
  if (k % 2 == 1) {
    const int off = (k - 1) / 2 - k;  // knots between data points
    for (int j = k + 1; j <= n; j++) t[j - 1] = R(0.5) * (x[off + j - 1] + x[off + j]);
  } else {
    const int off = k / 2 - k;  // knots at data points
    for (int j = k + 1; j <= n; j++) t[j - 1] = x[off + j - 1];
  }
}

// the k basis values of order k that are non-zero on [t(l), t(l+1)) at xv (l 1-based)
template <typename R>
static void basis(const std::vector<R> &t, int k, int l, R xv, R *b) {
  R dr[8], dl[8];
  b[0] = R(1);
  for (int j = 1; j < k; j++) {
    dr[j] = t[l + j - 1] - xv;
    dl[j] = xv - t[l - j];
    R prev = R(0);
    for (int m = 1; m <= j; m++) {
      const R vm = b[m - 1] / (dr[m] + dl[j + 1 - m]);
      b[m - 1] = vm * dr[m] + prev;
      prev = vm * dl[j + 1 - m];
    }
    b[j] = prev;
  }
}

template <typename R>
bool SplineAxisHost<R>::build(const std::vector<R> &x, int order) {
  n = (int)x.size();
  k = order;
  if (n < 3 || k < 2 || k >= n) return false;  // db3ink input checks (check_inputs)
  for (int i = 0; i + 1 < n; i++)
    if (!(x[i] < x[i + 1])) return false;
  knots(x, n, k, t);
  const int nr = 2 * k - 1;
  lu.assign((size_t)nr * n, R(0));
  int left = k;
  for (int i = 1; i <= n; i++) {
    const R xi = x[i - 1];
    const int lim = std::min(i + k, n + 1);
    left = std::max(left, i);
    if (xi < t[left - 1]) return false;
    bool found = false;
    while (true) {
      if (xi < t[left]) {
        found = true;
        break;
      }
      left = left + 1;
      if (left >= lim) break;
    }
    if (!found) {
      left = left - 1;
      if (xi > t[left]) return false;
    }
    R b[8];
    basis(t, k, left, xi, b);
    for (int j = 1; j <= k; j++) {
      const int col = left - k + j;
      const int row = k + i - col;
      lu[(size_t)(row - 1) + (size_t)nr * (col - 1)] = b[j - 1];
    }
  }
  const int mid = k, nb = k - 1;
  auto W = [&](int r, int c) -> R & { return lu[(size_t)(r - 1) + (size_t)nr * (c - 1)]; };
  for (int i = 1; i <= n - 1; i++) {
    const R piv = W(mid, i);
    if (piv == R(0)) return false;
    const int jmax = std::min(nb, n - i);
    for (int j = 1; j <= jmax; j++) W(mid + j, i) = W(mid + j, i) / piv;
    const int kmax = std::min(nb, n - i);
    for (int kk = 1; kk <= kmax; kk++) {
      const int ipk = i + kk, midmk = mid - kk;
      const R fac = W(midmk, ipk);
      for (int j = 1; j <= jmax; j++) W(midmk + j, ipk) = W(midmk + j, ipk) - W(mid + j, i) * fac;
    }
  }
  if (W(mid, n) == R(0)) return false;
  // reciprocal spans per interval l: slot order j = 1..k-1, m = 1..j
  rinv.assign((size_t)(n + k) * 6, R(0));
  for (int l = k; l <= n; l++) {
    int slot = 0;
    for (int j = 1; j < k; j++)
      for (int m = 1; m <= j; m++) {
        const R span = t[l + m - 1] - t[l + m - j - 1];
        rinv[(size_t)(l - 1) * 6 + slot++] = span != R(0) ? R(1) / span : R(0);
      }
  }
  // intervals whose basis depends on equally spaced knots only, t(l-k+2) .. t(l+k-1): there
  // the k non-zero B-splines are the uniform polynomials of (x - t(l)) / h
  tu.assign((size_t)2 * (n + k), R(0));
  for (int l = 1; l <= n + k; l++) tu[(size_t)2 * (l - 1)] = t[l - 1];
  // (relative tolerance above the rounding of coordinates built as x0 + i dx; the uniform
  // polynomials then differ from the recurrence on the actual knots by about that much)
  const R tol = std::max(R(1e-9), R(64) * std::numeric_limits<R>::epsilon());
  for (int l = k; l <= n; l++) {
    const R h = t[l] - t[l - 1];
    if (!(h > R(0))) continue;
    bool uni = true;
    for (int m = l - k + 1; m + 1 <= l + k - 2; m++) {
      const R d = t[m + 1] - t[m];
      if (!(std::fabs(d - h) <= tol * h)) uni = false;
    }
    if (uni) tu[(size_t)2 * (l - 1) + 1] = R(1) / h;
  }
  return true;
}

template struct SplineAxisHost<double>;
template struct SplineAxisHost<float>;

}  // namespace cfd2lcs
