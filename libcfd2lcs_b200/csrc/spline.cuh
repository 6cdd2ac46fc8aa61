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

#include <type_traits>

#include "device_common.cuh"

namespace cfd2lcs {

template <typename T>
struct SplineAxis {
  int n;          // points along the axis (interior + 2 ghosts)
  int k;          // order (degree + 1)
  const T *t;     // n + k knots
  const T *rinv;  // per interval l (1-based, stored at l-1): 1/(t(l+r) - t(l+r-j)), 6 slots
  const T *pull;  // band LU of the collocation matrix in pull form, 8 values per element
  const T *tu;    // per interval l (pair at 2(l-1)): t(l) and 1/h where the knots are uniform, else 0
};

template <typename T>
struct Pair2;
template <>
struct Pair2<double> {
  using type = double2;
};
template <>
struct Pair2<float> {
  using type = float2;
};

template <typename T>
struct SplineAxes {
  SplineAxis<T> ax[3];
};

template <typename T>
struct SplineStencil {
  int p0;      // padded index of the first coefficient
  int c0[3];   // padded index of the first coefficient along each axis
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

// Which kernels take the uniform-knot basis below (the same values as the recurrence to
// rounding; kernels that must give each other's bits make the same choice): the backward
// semi-Lagrangian kernels, gathering and staged, when they gather FP32 velocity taps (the mixed
// form); the particle kernels -- the forward subcycle, gathering and staged, and the composition
// -- always.  Measured on B200 (ABC 256^3, RK3, cubic, FP64): the gathering forward kernel 6.63
// -> 6.32 ms per launch with it, the staged backward kernel 3.15 -> 3.18 ms.
template <typename T, typename TV>
__host__ __device__ constexpr bool uniform_basis() {
  return !std::is_same<T, TV>::value;
}
#ifndef CFD2LCS_PARTICLE_UNI
#define CFD2LCS_PARTICLE_UNI 1
#endif
__host__ __device__ constexpr bool particle_uniform_basis() { return CFD2LCS_PARTICLE_UNI != 0; }

// KC: the order when it is known at compile time for every axis (4 for cubic on a 3-D grid),
// 0 for the general case.  UNI: take the uniform-knot form where the knots allow it.
template <typename T, int KC, bool UNI = false>
__device__ __forceinline__ void basis_values(const SplineAxis<T> &A, int l, T x, T *b) {
  const int k = KC ? KC : A.k;
  // equally spaced knots (interior intervals of a uniform grid): the uniform B-spline
  // polynomials of u = (x - t(l)) / h -- the same values as the recurrence below to rounding,
  // from one paired table read instead of 3(k-1).  Chosen per kernel (uniform_basis,
  // particle_uniform_basis above).
  const typename Pair2<T>::type q =
      UNI ? __ldg(reinterpret_cast<const typename Pair2<T>::type *>(A.tu) + (l - 1)) : typename Pair2<T>::type{};
  const T iu = q.y;
  if (UNI && iu > T(0)) {
    const T u = (x - q.x) * iu, v = T(1) - u;
    if (k == 4) {
      const T s = T(1) / T(6), u2 = u * u, u3 = u2 * u;
      b[0] = s * (v * v * v);
      b[1] = s * (T(3) * u3 - T(6) * u2 + T(4));
      b[2] = s * (T(-3) * u3 + T(3) * u2 + T(3) * u + T(1));
      b[3] = s * u3;
      return;
    }
    if (k == 3) {
      const T s = T(1) / T(2), u2 = u * u;
      b[0] = s * (v * v);
      b[1] = s * (T(-2) * u2 + T(2) * u + T(1));
      b[2] = s * u2;
      return;
    }
    if (k == 2) {
      b[0] = v;
      b[1] = u;
      return;
    }
  }
  // Cox-de Boor recurrence with the reciprocal knot spans of interval l
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
template <typename T, int KC, bool UNI = false>
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
    basis_values<T, KC, UNI>(A, l, x[a], st.b[a]);
    c0[a] = l - k;  // padded index of coefficient l-k+1 (1-based)
    st.c0[a] = c0[a];
  }
  st.p0 = pidx(g.P.sx, g.P.sxy, c0[0], c0[1], c0[2]);
  return true;
}

// Tensor contraction of the k x k x k coefficients around the stencil, x then y then z.
// TC is the coefficient type: the mixed-precision form contracts FP32 velocity coefficients
// with the basis values rounded to FP32.  tap(c1, c2, c0) returns coefficient (c0, c1, c2)
// of the stencil: from global memory (spline_apply) or from a tile staged in shared memory
// (the tiled backward kernel) -- one FMA sequence for both, so both give the same bits.
template <typename T, int KC, typename TC, typename Tap>
__device__ __forceinline__ TC spline_contract(const SplineAxes<T> &S, const SplineStencil<T> &st, Tap tap) {
  const int kx = KC ? KC : S.ax[0].k, ky = KC ? KC : S.ax[1].k, kz = KC ? KC : S.ax[2].k;
  TC vz = TC(0);
#pragma unroll
  for (int c2 = 0; c2 < 4; c2++) {
    if (c2 >= kz) break;
    TC vy = TC(0);
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) {
      if (c1 >= ky) break;
      TC vx = TC(0);
#pragma unroll
      for (int c0 = 0; c0 < 4; c0++) {
        if (c0 >= kx) break;
        vx += TC(st.b[0][c0]) * tap(c1, c2, c0);
      }
      vy += TC(st.b[1][c1]) * vx;
    }
    vz += TC(st.b[2][c2]) * vy;
  }
  return vz;
}

template <typename T, int KC, typename TC = T>
__device__ __forceinline__ TC spline_apply(const DevGrid<T> &g, const SplineAxes<T> &S, const SplineStencil<T> &st,
                                           const TC *__restrict__ coef) {
  const int sx = g.P.sx, sxy = g.P.sxy, p0 = st.p0;
  return spline_contract<T, KC, TC>(S, st, [&](int c1, int c2, int c0) { return __ldg(coef + p0 + c1 * sx + c2 * sxy + c0); });
}

// ---------------------------------------------------------------------------------------
// Banded solve of one line in place (dbnslv, src/bspline/bspline_sub_module.f90:2202-2259):
// forward elimination with the unit lower factor, then back substitution.
// ---------------------------------------------------------------------------------------
// Banded substitutions of the collocation LU (dbnfac / dbnslv, src/bspline/
// bspline_sub_module.f90:2098-2259) in pull form.  For element i (1-based) the host stores
//   pull[8(i-1) + j-1]     = L(i, i-j) = W(mid+j, i-j)   j = 1..k-1  (0 where i-j < 1)
//   pull[8(i-1) + 3 + j-1] = U(i, i+j) = W(mid-j, i+j)   j = 1..k-1  (0 where i+j > n)
//   pull[8(i-1) + 6]       = 1 / W(mid, i)
// Forward: x(i) = b(i) - L(i,i-k+1) x(i-k+1) - ... - L(i,i-1) x(i-1), the updates in the order
// in which dbnslv's row-by-row elimination applies them.  Backward: x(i) = (b(i) - U(i,i+k-1)
// x(i+k-1) - ... - U(i,i+1) x(i+1)) * (1 / W(mid,i)).  Each element needs only the k-1
// solved neighbours before it, kept in registers, so a line streams through once per sweep.
// win[0] holds the nearest solved neighbour.
template <typename T, int K>
__device__ __forceinline__ T pull_forward(const T *__restrict__ pc, int i0, T b, T (&win)[3]) {
  const T *c = pc + 8 * i0;  // i0 = i - 1
#pragma unroll
  for (int j = K - 1; j >= 1; j--) b = b - win[j - 1] * __ldg(c + j - 1);
  win[2] = win[1];
  win[1] = win[0];
  win[0] = b;
  return b;
}

template <typename T, int K>
__device__ __forceinline__ T pull_backward(const T *__restrict__ pc, int i0, T b, T (&win)[3]) {
  const T *c = pc + 8 * i0;
#pragma unroll
  for (int j = K - 1; j >= 1; j--) b = b - win[j - 1] * __ldg(c + 3 + j - 1);
  b = b * __ldg(c + 6);
  win[2] = win[1];
  win[1] = win[0];
  win[0] = b;
  return b;
}

}  // namespace cfd2lcs
