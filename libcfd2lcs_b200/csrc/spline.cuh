// Tensor-product B-spline interpolation on the ghost-padded grid, the QUADRATIC / CUBIC
// interpolators of interp_s2u_r1 (src/lp_tracking_m.f90:476-524), which call the vendored
// bspline-fortran (src/bspline/bspline_sub_module.f90).
//
// Fit: the reference fits a not-a-knot interpolating spline over the whole padded array
// (db3ink :451-533: knots by dbknot :1737-1785, one banded collocation solve per line along
// x, then y, then z, dbtpcf/dbintk/dbnfac/dbnslv :1801-2259).  The collocation matrix of an
// axis depends only on the grid, so its LU factors are computed once on the host
// (spline_host.cpp) and the device only runs the banded forward/back substitutions.
//
// Evaluation: db3val (:574-656) returns 0 outside [t(1), t(n+k)] and when the y or z
// interval search reports x >= t(n+k); an x exactly at the right end takes the left limit
// (dbvalu :2397-2533).  The value is the same polynomial as de Boor's recurrence, formed
// here from the k non-zero basis values per axis (Cox-de Boor, as dbspvn :2288-2370).
#pragma once

#include "device_common.cuh"

namespace cfd2lcs {

template <typename T>
struct SplineAxis {
  int n;          // points along the axis (interior + 2 ghosts)
  int k;          // order (degree + 1)
  const T *t;     // n + k knots
  const T *rinv;  // per interval l (1-based, stored at l-1): 1/(t(l+r) - t(l+r-j)), 6 slots
  const T *lu;    // band LU of the collocation matrix, (2k-1) x n column-major
};

template <typename T>
struct SplineAxes {
  SplineAxis<T> ax[3];
};

template <typename T>
struct SplineStencil {
  int p0;      // padded index of the first coefficient
  T b[3][4];   // basis values per axis (only the first k used)
};

// largest l (1-based) in [lo, hi] with t(l) <= x, walking from a guess (t(lo) <= x holds).
// Departure points and tracked particles sit within a cell or two of their node, so the
// walk is short; it is exact for any guess.
template <typename T>
__device__ __forceinline__ int knot_interval(const T *t, T x, int lo, int hi, int guess) {
  int l = min(max(guess, lo), hi);
  while (l < hi && __ldg(t + l) <= x) l++;      // t(l+1) <= x
  while (l > lo && __ldg(t + l - 1) > x) l--;   // t(l) > x
  return l;
}

// KC: the order when it is known at compile time for every axis (4 for cubic on a 3-D grid),
// 0 for the general case.
template <typename T, int KC>
__device__ __forceinline__ void basis_values(const SplineAxis<T> &A, int l, T x, T *b) {
  // Cox-de Boor recurrence with the reciprocal knot spans of interval l
  const int k = KC ? KC : A.k;
  const T *r = A.rinv + (size_t)(l - 1) * 6;
  T dr[4], dl[4];
  b[0] = T(1);
  int slot = 0;
#pragma unroll
  for (int j = 1; j < 4; j++) {
    if (j >= k) break;
    dr[j] = __ldg(A.t + l + j - 1) - x;  // t(l+j) - x
    dl[j] = x - __ldg(A.t + l - j);      // x - t(l+1-j)
    T prev = T(0);
#pragma unroll
    for (int m = 1; m <= 3; m++) {
      if (m > j) break;
      const T vm = b[m - 1] * __ldg(r + slot++);  // b / (t(l+m) - t(l+m-j))
      b[m - 1] = vm * dr[m] + prev;
      prev = vm * dl[j + 1 - m];
    }
    b[j] = prev;
  }
}

// Locates x in the padded spline; false where db3val returns 0.  no[] is the padded node
// the point belongs to (its interval is near no + k - 1).
template <typename T, int KC>
__device__ __forceinline__ bool spline_stencil(const DevGrid<T> &g, const SplineAxes<T> &S, const T x[3], const int no[3],
                                               SplineStencil<T> &st) {
  int c0[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const SplineAxis<T> &A = S.ax[a];
    const int n = A.n, k = KC ? KC : A.k;
    const T tfirst = __ldg(A.t), tlast = __ldg(A.t + n + k - 1);
    if (!(x[a] >= tfirst) || x[a] > tlast) return false;
    int l;
    if (a == 0) {
      // dbvalu's search over t(1..n+1); x == t(n+1) takes the left limit at interval n
      l = (x[a] >= __ldg(A.t + n)) ? n : knot_interval(A.t, x[a], k, n, no[a] + k - 1);
    } else {
      // db3val's search over the whole knot vector; x >= t(n+k) gives 0
      if (x[a] >= tlast) return false;
      l = knot_interval(A.t, x[a], k, n, no[a] + k - 1);
    }
    basis_values<T, KC>(A, l, x[a], st.b[a]);
    c0[a] = l - k;  // padded index of coefficient l-k+1 (1-based)
  }
  st.p0 = pidx(g.P.sx, g.P.sxy, c0[0], c0[1], c0[2]);
  return true;
}

template <typename T, int KC>
__device__ __forceinline__ T spline_apply(const DevGrid<T> &g, const SplineAxes<T> &S, const SplineStencil<T> &st,
                                          const T *__restrict__ coef) {
  const int kx = KC ? KC : S.ax[0].k, ky = KC ? KC : S.ax[1].k, kz = KC ? KC : S.ax[2].k;
  T vz = T(0);
#pragma unroll
  for (int c2 = 0; c2 < 4; c2++) {
    if (c2 >= kz) break;
    T vy = T(0);
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) {
      if (c1 >= ky) break;
      const T *row = coef + st.p0 + c1 * g.P.sx + c2 * g.P.sxy;
      T vx = T(0);
#pragma unroll
      for (int c0 = 0; c0 < 4; c0++) {
        if (c0 >= kx) break;
        vx += st.b[0][c0] * __ldg(row + c0);
      }
      vy += st.b[1][c1] * vx;
    }
    vz += st.b[2][c2] * vy;
  }
  return vz;
}

// ---------------------------------------------------------------------------------------
// Banded solve of one line in place (dbnslv, src/bspline/bspline_sub_module.f90:2202-2259):
// forward elimination with the unit lower factor, then back substitution.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void band_solve_line(const SplineAxis<T> &A, T *b, long stride) {
  const int n = A.n, k = A.k, nr = 2 * k - 1, mid = k;  // mid is 1-based
  const T *w = A.lu;
#define Wm(r, c) __ldg(w + ((r)-1) + (size_t)nr * ((c)-1))
#define Bm(i) b[(long)((i)-1) * stride]
  if (n != 1) {
    for (int i = 1; i <= n - 1; i++) {
      const T bi = Bm(i);
      const int jmax = min(k - 1, n - i);
      for (int j = 1; j <= jmax; j++) Bm(i + j) = Bm(i + j) - bi * Wm(mid + j, i);
    }
    for (int i = n; i >= 2; i--) {
      const T bi = Bm(i) / Wm(mid, i);
      Bm(i) = bi;
      const int jmax = min(k - 1, i - 1);
      for (int j = 1; j <= jmax; j++) Bm(i - j) = Bm(i - j) - bi * Wm(mid - j, i);
    }
  }
  Bm(1) = Bm(1) / Wm(mid, 1);
#undef Wm
#undef Bm
}

// Same solve with a register window of k values per pass: every element is loaded and
// stored once in the forward and once in the backward pass, and receives its updates in the
// reference's order (forward: from rows i = m-k+1 .. m-1; backward: from i = m+k-1 .. m+1).
template <typename T, int K>
__device__ __forceinline__ void band_solve_window(const SplineAxis<T> &A, T *b, long stride) {
  const int n = A.n, nr = 2 * K - 1, mid = K;
  const T *w = A.lu;
#define Wm(r, c) __ldg(w + ((r)-1) + (size_t)nr * ((c)-1))
  T win[K];
  if (n == 1) {
    b[0] = b[0] / Wm(mid, 1);
    return;
  }
  // forward elimination: window holds b(i) .. b(i+K-1)
#pragma unroll
  for (int q = 0; q < K; q++) win[q] = (q < n) ? b[(long)q * stride] : T(0);
  for (int i = 1; i <= n - 1; i++) {
    const T bi = win[0];
    b[(long)(i - 1) * stride] = bi;
#pragma unroll
    for (int j = 1; j < K; j++)
      if (i + j <= n) win[j] = win[j] - bi * Wm(mid + j, i);
#pragma unroll
    for (int q = 0; q < K - 1; q++) win[q] = win[q + 1];
    win[K - 1] = (i + K <= n) ? b[(long)(i + K - 1) * stride] : T(0);
  }
  b[(long)(n - 1) * stride] = win[0];
  // back substitution: window holds b(i), b(i-1), .., b(i-K+1)
#pragma unroll
  for (int q = 0; q < K; q++) win[q] = (n - q >= 1) ? b[(long)(n - 1 - q) * stride] : T(0);
  for (int i = n; i >= 2; i--) {
    const T bi = win[0] / Wm(mid, i);
    b[(long)(i - 1) * stride] = bi;
#pragma unroll
    for (int j = 1; j < K; j++)
      if (i - j >= 1) win[j] = win[j] - bi * Wm(mid - j, i);
#pragma unroll
    for (int q = 0; q < K - 1; q++) win[q] = win[q + 1];
    win[K - 1] = (i - K >= 1) ? b[(long)(i - K - 1) * stride] : T(0);
  }
  b[0] = win[0] / Wm(mid, 1);
#undef Wm
}

}  // namespace cfd2lcs
