// Point-wise advection pieces shared by the backward semi-Lagrangian kernel, the forward
// particle kernel and the composition kernel: interpolation stencils (NEAREST, LINEAR,
// B-spline), the five Runge-Kutta integrators with the reference's stage placement,
// boundary conditions on particles and the node search.
#pragma once

#include <type_traits>

#include "device_common.cuh"
#include "spline.cuh"

namespace cfd2lcs {

// product and sum rounded on their own (never contracted into an FMA), as the reference's
// compiled arithmetic forms them
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// The interpolation fraction a / b of a LINEAR stencil from y = RN(1 / b), the bracket's
// reciprocal span taken from a table: Markstein's correction step (P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990),
// q0 = RN(a y), r = a - b q0 (exact in one FMA), q = RN(q0 + r y).  With a correctly rounded
// reciprocal and q0 within one ulp of a / b, q is the correctly rounded quotient; it replaces
// the IEEE division on the stencils' dependent chain.  Every LINEAR stencil of the library forms
// its fraction this way, so the staged and gathering kernels stay bitwise equal to each other.
template <typename T>
__device__ __forceinline__ T lin_quotient(T a, T b, T y) {
  const T q0 = mul_rn(a, y);
  const T r = fma_rn(-b, q0, a);
  return fma_rn(r, y, q0);
}
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// ---------------------------------------------------------------------------------------
// Trilinear stencil around a node, interp_s2u_r1 LINEAR (src/lp_tracking_m.f90:342-474):
// per axis the bracket is [no, no+1] when x > line(no), else [no-1, no]; t is clamped to
// [0,1]; the eight weights are formed as mt*mt*mt ... in the reference's order.
// ---------------------------------------------------------------------------------------
template <typename T>
struct LinStencil {
  int p0;         // padded index of the lower corner
  int s[3];       // padded stride of the upper corner along each axis (0 if clamped onto p0)
  int i0[3];      // padded index of the lower corner along each axis
  int d[3];       // 1 where the upper corner differs from the lower one, else 0
  T w[8];
};

template <typename T>
__device__ __forceinline__ void lin_stencil(const DevGrid<T> &g, const T x[3], const int no[3], LinStencil<T> &st) {
  int i0[3];
  T t[3], mt[3];
  const int str[3] = {1, g.P.sx, g.P.sxy};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const T *L = g.li[a];
    const int n0 = no[a];
    int lo, hi;
    if (x[a] > __ldg(L + n0)) {
      lo = n0;
      hi = n0 + 1;
    } else {
      lo = n0 - 1;
      hi = n0;
    }
    // the reference leaves a bracket outside the padded array undefined; keep it inside
    lo = min(max(lo, 0), g.P.n[a] + 1);
    hi = min(max(hi, 0), g.P.n[a] + 1);
    const T x0 = __ldg(L + lo), x1 = __ldg(L + hi);
    // a bracket clamped onto one line (hi == lo) keeps the IEEE division of its 0 span
    t[a] = clamp01(hi > lo && g.ri[a] ? lin_quotient(x[a] - x0, x1 - x0, __ldg(g.ri[a] + lo)) : (x[a] - x0) / (x1 - x0));
    mt[a] = T(1) - t[a];
    i0[a] = lo;
    st.i0[a] = lo;
    st.d[a] = hi - lo;
    st.s[a] = (hi - lo) * str[a];
  }
  st.p0 = pidx(g.P.sx, g.P.sxy, i0[0], i0[1], i0[2]);
  st.w[0] = mt[0] * mt[1] * mt[2];
  st.w[1] = t[0] * mt[1] * mt[2];
  st.w[2] = mt[0] * t[1] * mt[2];
  st.w[3] = t[0] * t[1] * mt[2];
  st.w[4] = mt[0] * mt[1] * t[2];
  st.w[5] = t[0] * mt[1] * t[2];
  st.w[6] = mt[0] * t[1] * t[2];
  st.w[7] = t[0] * t[1] * t[2];
}

// lin_stencil around a grid node no (1 <= no <= n on every axis) from the node's interpolation
// lines lm, lc, lp at no-1, no, no+1 and the reciprocal spans rm = ri[no-1], rp = ri[no]: the
// bracket is [no, no+1] or [no-1, no], which the clamps of lin_stencil leave as they are, so the
// stencil is the same in every bit.
template <typename T>
__device__ __forceinline__ void lin_stencil_node(const T lm[3], const T lc[3], const T lp[3], const T rm[3], const T rp[3], int sx, int sxy,
                                                 const T x[3], const int no[3], LinStencil<T> &st) {
  const int str[3] = {1, sx, sxy};
  T t[3], mt[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const bool up = x[a] > lc[a];
    const T x0 = up ? lc[a] : lm[a], x1 = up ? lp[a] : lc[a];
    t[a] = clamp01(lin_quotient(x[a] - x0, x1 - x0, up ? rp[a] : rm[a]));
    mt[a] = T(1) - t[a];
    st.i0[a] = up ? no[a] : no[a] - 1;
    st.d[a] = 1;
    st.s[a] = str[a];
  }
  st.p0 = pidx(sx, sxy, st.i0[0], st.i0[1], st.i0[2]);
  st.w[0] = mt[0] * mt[1] * mt[2];
  st.w[1] = t[0] * mt[1] * mt[2];
  st.w[2] = mt[0] * t[1] * mt[2];
  st.w[3] = t[0] * t[1] * mt[2];
  st.w[4] = mt[0] * mt[1] * t[2];
  st.w[5] = t[0] * mt[1] * t[2];
  st.w[6] = mt[0] * t[1] * t[2];
  st.w[7] = t[0] * t[1] * t[2];
}

// Corner c of the stencil (bit 0: x, bit 1: y, bit 2: z upper corner) as a padded index; the
// contractions below take the corner values through a loader, so the gathering kernels and the
// shared-memory tile kernels run one expression (and get the same bits).
template <typename T>
__device__ __forceinline__ int lin_corner(const LinStencil<T> &st, int c) {
  return st.p0 + ((c & 1) ? st.s[0] : 0) + ((c & 2) ? st.s[1] : 0) + ((c & 4) ? st.s[2] : 0);
}

template <typename T, typename V>
__device__ __forceinline__ T lin_contract(const LinStencil<T> &st, V v) {
  return st.w[0] * v(0) + st.w[1] * v(1) + st.w[2] * v(2) + st.w[3] * v(3) + st.w[4] * v(4) + st.w[5] * v(5) + st.w[6] * v(6) +
         st.w[7] * v(7);
}

template <typename T>
__device__ __forceinline__ T lin_apply(const LinStencil<T> &st, const T *__restrict__ f) {
  return lin_contract<T>(st, [&](int c) { return __ldg(f + lin_corner(st, c)); });
}

// time-blended field u = (1-ct) u_n + ct u_np1 at the corners, then trilinear; TV is the
// velocity storage type (FP32 in the mixed-precision form, weights rounded to it).  va(c), vb(c)
// return corner c of u_n and u_np1.
template <typename T, typename TV, typename VA, typename VB>
__device__ __forceinline__ TV lin_blend_contract(const LinStencil<T> &st, TV omc, TV ct, VA va, VB vb) {
  TV acc = TV(0);
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const TV v = omc * va(c) + ct * vb(c);
    acc = c == 0 ? TV(st.w[0]) * v : acc + TV(st.w[c]) * v;
  }
  return acc;
}

template <typename T, typename TV>
__device__ __forceinline__ TV lin_apply_blend(const LinStencil<T> &st, const TV *__restrict__ a, const TV *__restrict__ b, TV omc,
                                              TV ct) {
  return lin_blend_contract<T, TV>(st, omc, ct, [&](int c) { return __ldg(a + lin_corner(st, c)); },
                                   [&](int c) { return __ldg(b + lin_corner(st, c)); });
}

// a stage's time blend written beforehand (k_blend), sampled trilinearly with the same weights
// and accumulation as lin_apply_blend
template <typename T, typename TV>
__device__ __forceinline__ TV lin_apply_tv(const LinStencil<T> &st, const TV *__restrict__ f) {
  TV acc = TV(0);
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const TV v = __ldg(f + lin_corner(st, c));
    acc = c == 0 ? TV(st.w[0]) * v : acc + TV(st.w[c]) * v;
  }
  return acc;
}

// ---------------------------------------------------------------------------------------
// Taylor series about the tracked node, interp_s2u_r1 TSE / TSE_LIMIT
// (src/lp_tracking_m.f90:526-654), on this library's rectilinear grids:
//   phi(x) = phi(no) + grad(phi)(no) . (x - x(no)),
// grad by grad_sr1's second-order central differences over the node coordinates
// (src/gradient_m.f90:11-66), which the reference evaluates at interior nodes only (the
// gradient array stays zero on the ghost layer) and zeroes along a singleton axis; the
// three terms are added in the reference's order, each product and sum rounded on its own.
// TSE_LIMIT then clamps the value to the range of the 27 values around no (max with the
// minimum first, then min with the maximum).  At a ghost node that window reaches past the
// padded array -- the reference reads outside its allocation there -- and is clipped to it.
// val(p) returns the sampled field at padded index p in T.
// ---------------------------------------------------------------------------------------
template <typename T, bool LIMIT, typename F>
__device__ __forceinline__ T tse_apply(const DevGrid<T> &g, const T x[3], const int no[3], F val) {
  const int str[3] = {1, g.P.sx, g.P.sxy};
  const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
  const T v0 = val(p);
  T r = v0;
  const bool interior = no[0] >= 1 && no[0] <= g.P.n[0] && no[1] >= 1 && no[1] <= g.P.n[1] && no[2] >= 1 && no[2] <= g.P.n[2];
  if (interior) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (g.P.n[a] == 1) continue;
      const T *L = g.lt[a];
      const T d = (val(p + str[a]) - val(p - str[a])) / (__ldg(L + no[a] + 1) - __ldg(L + no[a] - 1));
      r = add_rn(r, mul_rn(x[a] - __ldg(L + no[a]), d));
    }
  }
  if (LIMIT) {
    T mn = v0, mx = v0;
    const int i0 = max(no[0] - 1, 0), i1 = min(no[0] + 1, g.P.n[0] + 1);
    const int j0 = max(no[1] - 1, 0), j1 = min(no[1] + 1, g.P.n[1] + 1);
    const int k0 = max(no[2] - 1, 0), k1 = min(no[2] + 1, g.P.n[2] + 1);
    for (int k = k0; k <= k1; k++)
      for (int j = j0; j <= j1; j++)
        for (int i = i0; i <= i1; i++) {
          const T v = val(pidx(g.P.sx, g.P.sxy, i, j, k));
          mn = v < mn ? v : mn;
          mx = v > mx ? v : mx;
        }
    r = r < mn ? mn : r;
    r = r > mx ? mx : r;
  }
  return r;
}

// Coordinates of padded node (i,j,k): the full arrays of a non-rectilinear grid (CURV), else
// the coordinate lines.
template <typename T, bool CURV>
__device__ __forceinline__ void node_xyz(const DevGrid<T> &g, int i, int j, int k, T x[3]) {
  if (CURV) {
    const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
#pragma unroll
    for (int a = 0; a < 3; a++) x[a] = __ldg(g.X[a] + p);
  } else {
    x[0] = __ldg(g.lt[0] + i);
    x[1] = __ldg(g.lt[1] + j);
    x[2] = __ldg(g.lt[2] + k);
  }
}

// ---------------------------------------------------------------------------------------
// Taylor series on a non-rectilinear grid, interp_s2u_r1 TSE / TSE_LIMIT with grad_sr1_ls
// (src/lp_tracking_m.f90:526-654, src/gradient_m.f90:241-295): at an interior node the
// gradient sums, over the six face neighbours in NBR_OFFSET order (2..7), (phi(nbr) -
// phi(no)) times the node's least-squares weights, from zero; on the ghost layer it is zero.
// The value is phi(no) + d_x g_x + d_y g_y + d_z g_z with d = x - x(no), left to right, every
// product and sum rounded on its own.  TSE_LIMIT clamps as tse_apply does.
// ---------------------------------------------------------------------------------------
template <typename T, bool LIMIT, typename F>
__device__ __forceinline__ T tse_ls_apply(const DevGrid<T> &g, const T x[3], const int no[3], F val) {
  const int str[3] = {1, g.P.sx, g.P.sxy};
  const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
  const T v0 = val(p);
  const bool interior = no[0] >= 1 && no[0] <= g.P.n[0] && no[1] >= 1 && no[1] <= g.P.n[1] && no[2] >= 1 && no[2] <= g.P.n[2];
  T gr[3] = {T(0), T(0), T(0)};
  if (interior) {
    const size_t plane = (size_t)g.P.sxy * (g.P.n[2] + 2);
#pragma unroll
    for (int nb = 0; nb < 6; nb++) {
      const int a = nb % 3, q = nb < 3 ? p - str[a] : p + str[a];
      const T df = val(q) - v0;
#pragma unroll
      for (int c = 0; c < 3; c++) gr[c] = add_rn(gr[c], mul_rn(df, __ldg(g.lsw + (size_t)(nb * 3 + c) * plane + p)));
    }
  }
  T r = v0;
#pragma unroll
  for (int a = 0; a < 3; a++) r = add_rn(r, mul_rn(x[a] - __ldg(g.X[a] + p), gr[a]));
  if (LIMIT) {
    T mn = v0, mx = v0;
    const int i0 = max(no[0] - 1, 0), i1 = min(no[0] + 1, g.P.n[0] + 1);
    const int j0 = max(no[1] - 1, 0), j1 = min(no[1] + 1, g.P.n[1] + 1);
    const int k0 = max(no[2] - 1, 0), k1 = min(no[2] + 1, g.P.n[2] + 1);
    for (int k = k0; k <= k1; k++)
      for (int j = j0; j <= j1; j++)
        for (int i = i0; i <= i1; i++) {
          const T v = val(pidx(g.P.sx, g.P.sxy, i, j, k));
          mn = v < mn ? v : mn;
          mx = v > mx ? v : mx;
        }
    r = r < mn ? mn : r;
    r = r > mx ? mx : r;
  }
  return r;
}

// ---------------------------------------------------------------------------------------
// Velocity sampler for one stage: NEAREST, LINEAR or B-spline, blended in time.
// ---------------------------------------------------------------------------------------
template <typename T>
struct VelFields {  // T: velocity storage type
  const T *un[3];
  const T *unp1[3];
  // B-spline interpolators: coefficients of the time-blended velocity of each stage,
  // (1-ct) c(u_n) + ct c(u_np1) -- the spline of the blended field the reference fits per
  // stage (src/lp_motion_m.f90:193-197 then src/lp_tracking_m.f90:509-511), by linearity
  const T *cs[4][3];
};

// Positions and stencils in T (the position / flow-map type); velocity data in TV.  UNI: the
// uniform-knot basis for the B-splines (spline.cuh).
template <typename T, typename TV, int INTERP, bool UNI = uniform_basis<T, TV>()>
__device__ __forceinline__ void sample_velocity(const DevGrid<T> &g, const SplineAxes<T> &sa, const VelFields<TV> &V, const T x[3],
                                                const int no[3], T ct_, int stage, T out[3]) {
  const TV ct = TV(ct_);
  const TV omc = TV(1) - ct;
  if (INTERP == INTERP_NEAREST) {
    const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = T(omc * __ldg(V.un[c] + p) + ct * __ldg(V.unp1[c] + p));
  } else if (INTERP == INTERP_LINEAR) {
    LinStencil<T> st;
    lin_stencil(g, x, no, st);
    if (V.cs[stage][0]) {  // the stage's blend, written once per subcycle on large grids
#pragma unroll
      for (int c = 0; c < 3; c++) out[c] = T(lin_apply_tv<T, TV>(st, V.cs[stage][c]));
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) out[c] = T(lin_apply_blend<T, TV>(st, V.un[c], V.unp1[c], omc, ct));
    }
  } else if (INTERP == INTERP_TSE || INTERP == INTERP_TSE_LIMIT) {
    // the stage's field (1-ct) u_n + ct u_np1 at each node the expansion reads, as
    // integrate_lp blends the whole field before interpolating (src/lp_motion_m.f90:193-197)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const TV *a = V.un[c], *b = V.unp1[c];
      out[c] = tse_apply<T, INTERP == INTERP_TSE_LIMIT>(g, x, no, [&](int p) { return T(omc * __ldg(a + p) + ct * __ldg(b + p)); });
    }
  } else if (INTERP == INTERP_CTSE || INTERP == INTERP_CTSE_LIMIT) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const TV *a = V.un[c], *b = V.unp1[c];
      out[c] = tse_ls_apply<T, INTERP == INTERP_CTSE_LIMIT>(g, x, no, [&](int p) { return T(omc * __ldg(a + p) + ct * __ldg(b + p)); });
    }
  } else {
    constexpr int KC = INTERP == INTERP_SPLINE4 ? 4 : 0;
    SplineStencil<T> st;
    if (!spline_stencil<T, KC, UNI>(g, sa, x, no, st)) {
      out[0] = out[1] = out[2] = T(0);
      return;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = T(spline_apply<T, KC, TV>(g, sa, st, V.cs[stage][c]));
  }
}

// Velocity at a grid node, for a first stage that starts on the node (the backward SL
// subcycle): every interpolator reproduces the nodal data there -- NEAREST and LINEAR
// bitwise (the trilinear weights are exactly 0 and 1), the B-splines to rounding, since they
// interpolate the padded data at the abscissae, which are the node lines -- so the stage
// reads the two velocity levels at the node instead of the 64-tap stencil.
template <typename T, typename TV>
__device__ __forceinline__ void sample_velocity_node(const DevGrid<T> &g, const VelFields<TV> &V, const int no[3], T ct_, T out[3]) {
  const TV ct = TV(ct_);
  const TV omc = TV(1) - ct;
  const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
#pragma unroll
  for (int c = 0; c < 3; c++) out[c] = T(omc * __ldg(V.un[c] + p) + ct * __ldg(V.unp1[c] + p));
}

template <typename T, int INTERP, bool UNI = false>
__device__ __forceinline__ void sample_field(const DevGrid<T> &g, const SplineAxes<T> &sa, const T *const f[3], const T x[3],
                                             const int no[3], T out[3]) {
  if (INTERP == INTERP_NEAREST) {
    const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = __ldg(f[c] + p);
  } else if (INTERP == INTERP_LINEAR) {
    LinStencil<T> st;
    lin_stencil(g, x, no, st);
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = lin_apply(st, f[c]);
  } else if (INTERP == INTERP_TSE || INTERP == INTERP_TSE_LIMIT) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T *fc = f[c];
      out[c] = tse_apply<T, INTERP == INTERP_TSE_LIMIT>(g, x, no, [&](int p) { return __ldg(fc + p); });
    }
  } else if (INTERP == INTERP_CTSE || INTERP == INTERP_CTSE_LIMIT) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T *fc = f[c];
      out[c] = tse_ls_apply<T, INTERP == INTERP_CTSE_LIMIT>(g, x, no, [&](int p) { return __ldg(fc + p); });
    }
  } else {
    constexpr int KC = INTERP == INTERP_SPLINE4 ? 4 : 0;
    SplineStencil<T> st;
    if (!spline_stencil<T, KC, UNI>(g, sa, x, no, st)) {
      out[0] = out[1] = out[2] = T(0);
      return;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = spline_apply<T, KC>(g, sa, st, f[c]);
  }
}

// ---------------------------------------------------------------------------------------
// One integration step, integrate_lp (src/lp_motion_m.f90:129-360).  ct[] holds the stage
// time fractions the host computed for this subcycle (clamped, see stage_times()).
//   EULER       : ct[0]                    TRAPEZOIDAL: ct[0] = midpoint, velocity at xn
//   RK2         : ct[0] at t, ct[1] at t+dt/2
//   RK3         : ct[0] at t, ct[1] at t+dt/2, ct[2] at t+dt; stage 3 at xn + 2 k2
//   RK4         : ct[0] at t, ct[1] = ct[2] at t+dt/2, ct[3] at t+dt
// ---------------------------------------------------------------------------------------
struct StageTimes {
  double ct[4];
};

// AT_NODE: xn is the coordinate of node no (first stage by sample_velocity_node)
template <typename T, typename TV, int INTEG, int INTERP, bool AT_NODE = false, bool UNI = uniform_basis<T, TV>()>
__device__ __forceinline__ void integrate(const DevGrid<T> &g, const SplineAxes<T> &sa, const VelFields<TV> &V, const StageTimes &S,
                                          T dt, const T xn[3], const int no[3], T x[3]) {
  const T HALF = T(1) / T(2), THIRD = T(1) / T(3), TWOTHIRD = T(2) / T(3), SIXTH = T(1) / T(6), TWO = T(2);
  T u[3];
  auto first_stage = [&](T ct) {
    if (AT_NODE) sample_velocity_node<T, TV>(g, V, no, ct, u);
    else sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xn, no, ct, 0, u);
  };
  if (INTEG == EULER_ || INTEG == TRAPEZOIDAL_) {
    first_stage(T(S.ct[0]));
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = xn[c] + dt * u[c];
  } else if (INTEG == RK2_) {
    first_stage(T(S.ct[0]));
    T xh[3];
#pragma unroll
    for (int c = 0; c < 3; c++) xh[c] = xn[c] + HALF * dt * u[c];
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xh, no, T(S.ct[1]), 1, u);
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = xn[c] + dt * u[c];
  } else if (INTEG == RK3_) {
    T k[3], xs[3], acc[3];
    first_stage(T(S.ct[0]));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      acc[c] = xn[c] + SIXTH * k[c];
      xs[c] = xn[c] + HALF * k[c];
    }
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xs, no, T(S.ct[1]), 1, u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      xs[c] = xn[c] + TWO * k[c];
      acc[c] = acc[c] + TWOTHIRD * k[c];
    }
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xs, no, T(S.ct[2]), 2, u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * k[c];
    }
  } else {  // RK4
    T k[3], xs[3], acc[3];
    first_stage(T(S.ct[0]));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      acc[c] = xn[c] + SIXTH * k[c];
      xs[c] = xn[c] + HALF * k[c];
    }
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xs, no, T(S.ct[1]), 1, u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      acc[c] = acc[c] + THIRD * k[c];
      xs[c] = xn[c] + HALF * k[c];
    }
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xs, no, T(S.ct[2]), 2, u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      acc[c] = acc[c] + THIRD * k[c];
      xs[c] = xn[c] + k[c];
    }
    sample_velocity<T, TV, INTERP, UNI>(g, sa, V, xs, no, T(S.ct[3]), 3, u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * k[c];
    }
  }
}

// ---------------------------------------------------------------------------------------
// Particle boundary conditions.
// project_lp2plane (src/lp_m.f90:418-538) on a rectilinear 2-D grid: the plane normal is
// the singleton axis, so only that coordinate moves, x_a - (x_a - x_a(node)).
// set_lp_bc (src/lp_tracking_m.f90:185-277): the node is clamped to the interior; MASK
// nodes (and SLIP/WALL nodes on the boundary) project the particle back along bcnorm if
// it moved outward; INFLOW/OUTFLOW boundary nodes stick it to the node.
// Returns true when the particle sticks.
// ---------------------------------------------------------------------------------------
// (the singleton axis is selected by an unrolled comparison, not used as an index, so the
// position and node arrays stay in registers)
// On a non-rectilinear 2-D grid (CURV) the general form: the unit normal of the data plane at
// the clamped node, the distance (x - x(node)) . n, the normal turned to make it non-negative,
// and x - distance * n.
template <typename T, bool CURV = false>
__device__ __forceinline__ void project_plane(const DevGrid<T> &g, int no[3], T x[3]) {
  const int sa = g.P.single_axis;
  if (sa < 0) return;
  if constexpr (CURV) {
    no[0] = sa == 0 ? 1 : no[0];
    no[1] = sa == 1 ? 1 : no[1];
    no[2] = sa == 2 ? 1 : no[2];
    const int p = pidx(g.P.sx, g.P.sxy, min(max(no[0], 1), g.P.n[0]), min(max(no[1], 1), g.P.n[1]), min(max(no[2], 1), g.P.n[2]));
    T nv[3], d = T(0);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      nv[a] = __ldg(g.pnrm[a] + p);
      const T t = mul_rn(x[a] - __ldg(g.X[a] + p), nv[a]);
      d = a == 0 ? t : add_rn(d, t);
    }
    const bool flip = d < T(0);
    d = flip ? -d : d;
#pragma unroll
    for (int a = 0; a < 3; a++) x[a] = x[a] - mul_rn(d, flip ? -nv[a] : nv[a]);
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (a != sa) continue;
      no[a] = 1;
      const T plane = __ldg(g.lt[a] + 1);
      T d = x[a] - plane;
      const T dist = d < T(0) ? -d : d;
      const T nrm = d < T(0) ? T(-1) : T(1);
      x[a] = x[a] - dist * nrm;
    }
  }
}

template <typename T, bool HAS_FLAGS, bool CURV = false>
__device__ __forceinline__ bool particle_bc(const DevGrid<T> &g, int no[3], T x[3], int *err) {
#pragma unroll
  for (int a = 0; a < 3; a++) no[a] = min(max(no[a], 1), g.P.n[a]);
  if (!HAS_FLAGS) return false;
  const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
  const int f = g.flag[p];
  if (f == LCS_INTERNAL || f == LCS_2D) return false;
  const bool interior = no[0] > 1 && no[1] > 1 && no[2] > 1 && no[0] < g.P.n[0] && no[1] < g.P.n[1] && no[2] < g.P.n[2];
  if (f == LCS_MASK || f == LCS_SLIP || f == LCS_WALL) {
    if (f != LCS_MASK && interior) return false;
    T nx = __ldg(g.nrm[0] + p), ny = __ldg(g.nrm[1] + p), nz = __ldg(g.nrm[2] + p);
    T gn[3];
    node_xyz<T, CURV>(g, no[0], no[1], no[2], gn);
    const T gx = gn[0], gy = gn[1], gz = gn[2];
    const T dist = (x[0] - gx) * nx + (x[1] - gy) * ny + (x[2] - gz) * nz;
    if (dist > T(0)) {
      x[0] = x[0] - nx * dist;
      x[1] = x[1] - ny * dist;
      x[2] = x[2] - nz * dist;
    }
    return false;
  }
  if (f == LCS_INFLOW || f == LCS_OUTFLOW) {
    if (interior) return false;
    node_xyz<T, CURV>(g, no[0], no[1], no[2], x);
    return true;
  }
  atomicOr(err, ERR_UNKNOWN_FLAG);
  return false;
}

// ---------------------------------------------------------------------------------------
// Node search, track_lp2node (src/lp_tracking_m.f90:16-183): one pass looks at the 27
// neighbours (fewer on a 2-D grid) in NBR_OFFSET order (src/data_m.f90:124-152) and moves
// to one that is closer than 0.99 of the best so far.
// ---------------------------------------------------------------------------------------
// NBR_OFFSET as a constant expression; the search loop unrolls over it
__device__ __forceinline__ constexpr int nbr_offset(int nb, int a) {
  constexpr int8_t t[27][3] = {
      {0, 0, 0},   {-1, 0, 0},  {0, -1, 0}, {0, 0, -1}, {1, 0, 0},  {0, 1, 0},  {0, 0, 1},   {-1, -1, -1}, {0, -1, -1},
      {1, -1, -1}, {-1, 0, -1}, {1, 0, -1}, {-1, 1, -1}, {0, 1, -1}, {1, 1, -1}, {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},
      {1, 1, 0},   {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},  {-1, 0, 1}, {1, 0, 1},  {-1, 1, 1},  {0, 1, 1},   {1, 1, 1}};
  return t[nb][a];
}


// On a non-rectilinear grid (CURV) each candidate's squared distance comes from its padded
// coordinates, (gx - x)^2 + (gy - y)^2 + (gz - z)^2 rounded term by term, the candidate index
// clamped to the padded range.
template <typename T>
__device__ __forceinline__ bool track_pass_curv(const DevGrid<T> &g, const T x[3], int no[3]) {
  const int sa = g.P.single_axis;
  T best = T(0);
  bool have = false;
  int off[3] = {0, 0, 0};
#pragma unroll
  for (int nb = 0; nb < 27; nb++) {
    const int o0 = nbr_offset(nb, 0), o1 = nbr_offset(nb, 1), o2 = nbr_offset(nb, 2);
    if ((sa == 0 && o0 != 0) || (sa == 1 && o1 != 0) || (sa == 2 && o2 != 0)) continue;
    const int q = pidx(g.P.sx, g.P.sxy, min(max(no[0] + o0, 0), g.P.n[0] + 1), min(max(no[1] + o1, 0), g.P.n[1] + 1),
                       min(max(no[2] + o2, 0), g.P.n[2] + 1));
    const T e0 = __ldg(g.X[0] + q) - x[0], e1 = __ldg(g.X[1] + q) - x[1], e2 = __ldg(g.X[2] + q) - x[2];
    const T r = add_rn(add_rn(mul_rn(e0, e0), mul_rn(e1, e1)), mul_rn(e2, e2));
    if (!have || r < T(0.99) * best) {
      best = r;
      have = true;
      off[0] = o0;
      off[1] = o1;
      off[2] = o2;
    }
  }
  no[0] += off[0];
  no[1] += off[1];
  no[2] += off[2];
  return off[0] != 0 || off[1] != 0 || off[2] != 0;
}

template <typename T>
__device__ __forceinline__ bool track_pass_lines(const DevGrid<T> &g, const T x[3], int no[3]);

template <typename T, bool CURV = false>
__device__ __forceinline__ bool track_pass(const DevGrid<T> &g, const T x[3], int no[3]) {
  if constexpr (CURV) return track_pass_curv(g, x, no);
  else return track_pass_lines(g, x, no);
}

template <typename T>
__device__ __forceinline__ bool track_pass_lines(const DevGrid<T> &g, const T x[3], int no[3]) {
  // Per axis and offset o in {-1,0,1}: the squared axis distance to line no+o (clamped to
  // the padded range).  Off the interior the padded grid (sgrid%grid, src/sgrid_m.f90:
  // 182-359) holds one of two ghost coordinates: the periodic image when every out-of-range
  // axis of the candidate is periodic (sqp), the extrapolated one otherwise (sqn).  A
  // candidate's squared distance is then a sum of three register values; the 27 candidates
  // are unrolled with constant offsets.
  const int sa = g.P.single_axis;
  T sqp[3][3], sqn[3][3];
  unsigned ok = 0;  // bit 3a+o+1: line no[a]+o is interior, or axis a is periodic
#pragma unroll
  for (int a = 0; a < 3; a++) {
#pragma unroll
    for (int o = -1; o <= 1; o++) {
      const int v = min(max(no[a] + o, 0), g.P.n[a] + 1);
      const bool in = v >= 1 && v <= g.P.n[a];
      T cp, cn;
      if (in) {
        cp = cn = __ldg(g.lt[a] + v);
      } else {
        cp = v < 1 ? g.P.gx[a][0][1] : g.P.gx[a][1][1];
        cn = v < 1 ? g.P.gx[a][0][0] : g.P.gx[a][1][0];
      }
      const T dp = cp - x[a], dn = cn - x[a];
      sqp[a][o + 1] = mul_rn(dp, dp);
      sqn[a][o + 1] = mul_rn(dn, dn);
      if (in || g.P.per[a]) ok |= 1u << (3 * a + o + 1);
    }
  }
  T best = T(0);
  bool have = false;
  int off[3] = {0, 0, 0};
#pragma unroll
  for (int nb = 0; nb < 27; nb++) {
    const int o0 = nbr_offset(nb, 0), o1 = nbr_offset(nb, 1), o2 = nbr_offset(nb, 2);
    if ((sa == 0 && o0 != 0) || (sa == 1 && o1 != 0) || (sa == 2 && o2 != 0)) continue;
    const bool e = ((ok >> (o0 + 1)) & (ok >> (3 + o1 + 1)) & (ok >> (6 + o2 + 1)) & 1u) != 0;
    const T r = (e ? sqp[0][o0 + 1] : sqn[0][o0 + 1]) + (e ? sqp[1][o1 + 1] : sqn[1][o1 + 1]) +
                (e ? sqp[2][o2 + 1] : sqn[2][o2 + 1]);
    // rsq < 0.99*rsq_min with rsq_min starting at huge()
    if (!have || r < T(0.99) * best) {
      best = r;
      have = true;
      off[0] = o0;
      off[1] = o1;
      off[2] = o2;
    }
  }
  no[0] += off[0];
  no[1] += off[1];
  no[2] += off[2];
  return off[0] != 0 || off[1] != 0 || off[2] != 0;
}

// exchange_lpdata on one rank (src/comms_m.f90:872-1189): a particle whose node left the
// interior through a periodic direction is shifted by that direction's periodic shift and
// its node indices are wrapped.
template <typename T>
__device__ __forceinline__ void wrap_particle(const DevGrid<T> &g, T x[3], int no[3]) {
  int d[3];
#pragma unroll
  for (int a = 0; a < 3; a++) d[a] = no[a] < 1 ? -1 : (no[a] > g.P.n[a] ? 1 : 0);
  if (d[0] == 0 && d[1] == 0 && d[2] == 0) return;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (d[a] != 0 && !g.P.per[a]) return;
  const T *s = g.P.ps[(d[2] + 1) * 9 + (d[1] + 1) * 3 + (d[0] + 1)];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    x[a] = x[a] + s[a];
    int v = no[a];
    if (v > g.P.n[a]) v -= g.P.n[a];
    if (v < 1) v += g.P.n[a];
    no[a] = v;
  }
}

}  // namespace cfd2lcs
