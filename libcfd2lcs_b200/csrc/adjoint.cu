// Reverse-mode derivative of a backward-FTLE objective J = sum_x w(x) FTLE(x) with respect to
// the gridded velocity at every time level.  No counterpart in the reference library; the
// forward model is the library's own backward semi-Lagrangian path (update_flowmap_sl,
// src/flowmap_m.f90:17-104, with LINEAR interpolation, src/lp_tracking_m.f90:342-474, or the
// cubic B-spline, :476-524, and the steps of integrate_lp, src/lp_motion_m.f90:129-327) over every
// update from the first level to the last, and compute_ftle (src/lcs_m.f90:66-193) of the
// final flow map -- the frame the library computes when h equals the whole horizon.
//
// Forward: the velocity levels are ingested once (padded, ghost-filled, CFL maxima read back
// per level to fix every update's subcycle count); the flow map is stored every K updates
// (checkpoints).  Reverse: from the FTLE adjoint (eigenvector of the Cauchy-Green tensor,
// transpose of the central differences) back through every subcycle in reverse order; each
// checkpoint segment is first recomputed forward, keeping the flow map before each subcycle.
// The adjoint of one subcycle recomputes that subcycle's stage positions and scatters
// (atomicAdd) into the adjoint of the previous flow map and of the two velocity levels with
// the transposed trilinear weights; the position adjoint picks up the trilinear gradients.
// Ghost cells, which the forward fills as periodic copies, are folded back into their source
// nodes.  Discrete choices (subcycle counts, interpolation brackets, clamped weights) are
// held fixed, as differentiation of the piecewise-smooth map requires.
//
// Scope: a rectilinear grid with every flag LCS_INTERNAL and every non-singleton direction
// periodic (the ABC configuration); LINEAR or CUBIC interpolation (the cubic sweeps carry the
// adjoint through the spline fits); EULER, TRAPEZOIDAL, RK2, RK3 or RK4.
#include "adjoint.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "grid.h"
#include "kernels.cuh"
#include "spline_host.h"

namespace cfd2lcs {

namespace {

#define ACK(call)                                                                                \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      msg = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " + #call;               \
      return false;                                                                              \
    }                                                                                            \
  } while (0)

enum { EULER = 0, TRAPEZOIDAL = 1, RK2 = 2, RK3 = 3, RK4 = 4 };
enum { LINEAR_I = 1, CUBIC_I = 3 };

// device memory of one adjoint call
class Pool {
 public:
  ~Pool() {
    for (void *p : ptrs_) cudaFree(p);
  }
  template <typename X>
  X *alloc(size_t n, std::string &msg) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(X) > 0 ? n * sizeof(X) : 1);
    if (e != cudaSuccess) {
      msg = std::string("device allocation failed: ") + cudaGetErrorString(e);
      return nullptr;
    }
    ptrs_.push_back(p);
    return static_cast<X *>(p);
  }

 private:
  std::vector<void *> ptrs_;
};

// Trilinear stencil of lin_stencil (same brackets and clamped fractions) plus, per axis, the
// derivative of the fraction with respect to the coordinate (0 where the fraction is clamped).
template <typename T>
struct LinStencilAD {
  LinStencil<T> st;
  T t[3], dtdx[3];
};

template <typename T>
__device__ __forceinline__ void lin_stencil_ad(const DevGrid<T> &g, const T x[3], const int no[3], LinStencilAD<T> &s) {
  lin_stencil(g, x, no, s.st);
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
    lo = min(max(lo, 0), g.P.n[a] + 1);
    hi = min(max(hi, 0), g.P.n[a] + 1);
    const T x0 = __ldg(L + lo), x1 = __ldg(L + hi);
    const T raw = hi > lo && g.ri[a] ? lin_quotient(x[a] - x0, x1 - x0, __ldg(g.ri[a] + lo)) : (x[a] - x0) / (x1 - x0);
    s.t[a] = clamp01(raw);
    s.dtdx[a] = (raw > T(0) && raw < T(1)) ? T(1) / (x1 - x0) : T(0);
  }
}

// corner q (bit 0: x, bit 1: y, bit 2: z) of a trilinear stencil
template <typename T>
__device__ __forceinline__ int corner(const LinStencil<T> &st, int q) {
  return st.p0 + ((q & 1) ? st.s[0] : 0) + ((q & 2) ? st.s[1] : 0) + ((q & 4) ? st.s[2] : 0);
}

// d(weight_q)/d(t_a) of the trilinear weights
template <typename T>
__device__ __forceinline__ T dweight(const T t[3], int q, int a) {
  T r = T(1);
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const bool up = (q >> b) & 1;
    if (b == a) r *= up ? T(1) : T(-1);
    else r *= up ? t[b] : T(1) - t[b];
  }
  return r;
}

// particle_bc<T, true> (advect.cuh) for the particle of interior node no, recording what it did:
// a projection back along the boundary normal nrm (proj), or a stick to the node (returns true).
// The same arithmetic as the forward kernel, so the positions are its positions.
template <typename T>
__device__ __forceinline__ bool bc_record(const DevGrid<T> &g, const int no[3], T x[3], bool &proj, T nrm[3]) {
  proj = false;
  const int p = pidx(g.P.sx, g.P.sxy, no[0], no[1], no[2]);
  const int f = g.flag[p];
  if (f == LCS_INTERNAL || f == LCS_2D) return false;
  const bool interior = no[0] > 1 && no[1] > 1 && no[2] > 1 && no[0] < g.P.n[0] && no[1] < g.P.n[1] && no[2] < g.P.n[2];
  if (f == LCS_MASK || f == LCS_SLIP || f == LCS_WALL) {
    if (f != LCS_MASK && interior) return false;
    const T nx = __ldg(g.nrm[0] + p), ny = __ldg(g.nrm[1] + p), nz = __ldg(g.nrm[2] + p);
    const T gx = __ldg(g.lt[0] + no[0]), gy = __ldg(g.lt[1] + no[1]), gz = __ldg(g.lt[2] + no[2]);
    const T dist = (x[0] - gx) * nx + (x[1] - gy) * ny + (x[2] - gz) * nz;
    if (dist > T(0)) {
      x[0] = x[0] - nx * dist;
      x[1] = x[1] - ny * dist;
      x[2] = x[2] - nz * dist;
      proj = true;
      nrm[0] = nx;
      nrm[1] = ny;
      nrm[2] = nz;
    }
    return false;
  }
  if (f == LCS_INFLOW || f == LCS_OUTFLOW) return !interior;
  return false;
}

// The transpose of the plane projection and particle_bc on a position adjoint: zero after a
// stick, (I - n n^T) after a projection, the singleton axis' component dropped on a 2-D grid.
template <typename T>
__device__ __forceinline__ void bc_adjoint(const DevGrid<T> &g, bool stick, bool proj, const T nrm[3], T xb[3]) {
  if (stick) {
    xb[0] = xb[1] = xb[2] = T(0);
    return;
  }
  if (proj) {
    const T d = xb[0] * nrm[0] + xb[1] * nrm[1] + xb[2] * nrm[2];
#pragma unroll
    for (int c = 0; c < 3; c++) xb[c] -= nrm[c] * d;
  }
  const int sa = g.P.single_axis;
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (c == sa) xb[c] = T(0);
}

// ---------------------------------------------------------------------------------------
// Adjoint of one backward SL subcycle (k_sl_subcycle with LINEAR interpolation; F: boundary flags).
// fbn: adjoint of the new flow map (interior values used); fbo: accumulated adjoint of the
// previous map.  The velocity adjoint of the second stage goes to a2 (scattered, one blended
// field: the time blend is distributed onto the two levels afterwards by k_distribute), that
// of the first stage, which sits on the node, to a1 (plain stores).
// ---------------------------------------------------------------------------------------
// RK3 (integrate_lp, src/lp_motion_m.f90:212-263, with the third stage at xn + 2 k2): the
// third stage's velocity adjoint goes to a3 (scattered) and k_distribute takes its ct[2].
template <typename T, int INTEG, bool F = false>
__global__ void __launch_bounds__(256) k_sl_adjoint(DevGrid<T> g, VelFields<T> V, FieldPtrs<T> fmo, FieldPtrs<T> fbn, FieldPtrsW<T> fbo,
                                                     FieldPtrsW<T> a1, FieldPtrsW<T> a2, FieldPtrsW<T> a3, StageTimes S, T dt) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const T a[3] = {fbn.f[0][p], fbn.f[1][p], fbn.f[2][p]};
  if (a[0] == T(0) && a[1] == T(0) && a[2] == T(0)) return;
  const T HALF = T(1) / T(2);
  const int no[3] = {i, j, k};
  const T x0[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  // --- forward recomputation (integrate<>, first stage on the node) ---
  const T ct0 = T(S.ct[0]), omc0 = T(1) - ct0;
  T u1[3];
#pragma unroll
  for (int c = 0; c < 3; c++) u1[c] = omc0 * __ldg(V.un[c] + p) + ct0 * __ldg(V.unp1[c] + p);
  T x[3], xh[3], xs3[3], xs4[3];
  LinStencilAD<T> s2, s2b, s2c;
  const T ct1 = T(S.ct[1]), omc1 = T(1) - ct1;
  const T ct2 = T(S.ct[2]), omc2 = T(1) - ct2;
  const T ct3 = T(S.ct[3]), omc3 = T(1) - ct3;
  const T SIXTH = T(1) / T(6), TWOTHIRD = T(2) / T(3), TWO = T(2), THIRD = T(1) / T(3);
  if (INTEG == RK4) {
    // integrate_lp RK4 (src/lp_motion_m.f90:265-327): stages at xn + k1/2, xn + k2/2, xn + k3
    T k[3], acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u1[c];
      acc[c] = x0[c] + SIXTH * k[c];
      xh[c] = x0[c] + HALF * k[c];
    }
    lin_stencil_ad(g, xh, no, s2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * lin_apply_blend<T, T>(s2.st, V.un[c], V.unp1[c], omc1, ct1);
      acc[c] = acc[c] + THIRD * k[c];
      xs3[c] = x0[c] + HALF * k[c];
    }
    lin_stencil_ad(g, xs3, no, s2b);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * lin_apply_blend<T, T>(s2b.st, V.un[c], V.unp1[c], omc2, ct2);
      acc[c] = acc[c] + THIRD * k[c];
      xs4[c] = x0[c] + k[c];
    }
    lin_stencil_ad(g, xs4, no, s2c);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * lin_apply_blend<T, T>(s2c.st, V.un[c], V.unp1[c], omc3, ct3);
      x[c] = acc[c] + SIXTH * k[c];
    }
  } else if (INTEG == RK3) {
    T k[3], acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u1[c];
      acc[c] = x0[c] + SIXTH * k[c];
      xh[c] = x0[c] + HALF * k[c];
    }
    lin_stencil_ad(g, xh, no, s2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * lin_apply_blend<T, T>(s2.st, V.un[c], V.unp1[c], omc1, ct1);
      xs3[c] = x0[c] + TWO * k[c];
      acc[c] = acc[c] + TWOTHIRD * k[c];
    }
    lin_stencil_ad(g, xs3, no, s2b);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * lin_apply_blend<T, T>(s2b.st, V.un[c], V.unp1[c], omc2, ct2);
      x[c] = acc[c] + SIXTH * k[c];
    }
  } else if (INTEG == RK2) {
#pragma unroll
    for (int c = 0; c < 3; c++) xh[c] = x0[c] + HALF * dt * u1[c];
    lin_stencil_ad(g, xh, no, s2);
    T u2[3];
#pragma unroll
    for (int c = 0; c < 3; c++) u2[c] = lin_apply_blend<T, T>(s2.st, V.un[c], V.unp1[c], omc1, ct1);
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = x0[c] + dt * u2[c];
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = x0[c] + dt * u1[c];
  }
  // --- the forward kernel's plane projection and particle boundary condition ---
  bool stick = false, proj = false;
  T bn[3] = {T(0), T(0), T(0)};
  {
    int nb[3] = {i, j, k};
    project_plane(g, nb, x);
    if (F) stick = bc_record(g, nb, x, proj, bn);
    if (stick)
#pragma unroll
      for (int c = 0; c < 3; c++) x[c] = x0[c];
  }
  LinStencilAD<T> s3;
  lin_stencil_ad(g, x, no, s3);
  // --- fm_new = fm_old(x) + (x - x0) ---
  T xb[3] = {a[0], a[1], a[2]};
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int cq = corner(s3.st, q);
    const T wq = s3.st.w[q];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T f = __ldg(fmo.f[c] + cq);
      atomicAdd(fbo.f[c] + cq, wq * a[c]);
#pragma unroll
      for (int d = 0; d < 3; d++) xb[d] += a[c] * dweight(s3.t, q, d) * s3.dtdx[d] * f;
    }
  }
  bc_adjoint(g, stick, proj, bn, xb);
  // --- stages ---
  T u1b[3];
  // scatter of a sampled stage's velocity adjoint ub (weights of stencil st, blend omc/ct) into
  // a, returning the adjoint of the sample position in pb
  auto stage_back = [&](const LinStencilAD<T> &st, const T ub[3], FieldPtrsW<T> a, T omc, T ct, T pb[3]) {
    pb[0] = pb[1] = pb[2] = T(0);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int cq = corner(st.st, q);
      const T wq = st.st.w[q];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        atomicAdd(a.f[c] + cq, wq * ub[c]);
        const T vb = omc * __ldg(V.un[c] + cq) + ct * __ldg(V.unp1[c] + cq);
#pragma unroll
        for (int d = 0; d < 3; d++) pb[d] += ub[c] * dweight(st.t, q, d) * st.dtdx[d] * vb;
      }
    }
  };
  if (INTEG == RK4) {
    // x = xn + k1/6 + k2/3 + k3/3 + k4/6; the two half-step stages share ct and go to a2, the
    // last stage to a3 (distributed with ct[3])
    T k3b[3], k2b[3], k1b[3], ub[3], pb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k1b[c] = SIXTH * xb[c];
      k2b[c] = THIRD * xb[c];
      k3b[c] = THIRD * xb[c];
      ub[c] = dt * (SIXTH * xb[c]);
    }
    stage_back(s2c, ub, a3, omc3, ct3, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k3b[c] += pb[c];
      ub[c] = dt * k3b[c];
    }
    stage_back(s2b, ub, a2, omc2, ct2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k2b[c] += HALF * pb[c];
      ub[c] = dt * k2b[c];
    }
    stage_back(s2, ub, a2, omc1, ct1, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * (k1b[c] + HALF * pb[c]);
  } else if (INTEG == RK3) {
    // x = xn + k1/6 + 2 k2/3 + k3/6, k3 = dt u(xs3), xs3 = xn + 2 k2, k2 = dt u(xh), xh = xn + k1/2
    T k3b[3], k2b[3], k1b[3], ub[3], pb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k3b[c] = SIXTH * xb[c];
      k2b[c] = TWOTHIRD * xb[c];
      k1b[c] = SIXTH * xb[c];
      ub[c] = dt * k3b[c];
    }
    stage_back(s2b, ub, a3, omc2, ct2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k2b[c] += TWO * pb[c];
      ub[c] = dt * k2b[c];
    }
    stage_back(s2, ub, a2, omc1, ct1, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * (k1b[c] + HALF * pb[c]);
  } else if (INTEG == RK2) {
    T u2b[3], xhb[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int c = 0; c < 3; c++) u2b[c] = dt * xb[c];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int cq = corner(s2.st, q);
      const T wq = s2.st.w[q];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        atomicAdd(a2.f[c] + cq, wq * u2b[c]);
        const T vb = omc1 * __ldg(V.un[c] + cq) + ct1 * __ldg(V.unp1[c] + cq);
#pragma unroll
        for (int d = 0; d < 3; d++) xhb[d] += u2b[c] * dweight(s2.t, q, d) * s2.dtdx[d] * vb;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = HALF * dt * xhb[c];
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * xb[c];
  }
#pragma unroll
  for (int c = 0; c < 3; c++) a1.f[c][p] = u1b[c];
}

// velocity adjoint of one subcycle onto the two levels: un += (1-ct0) a1 + (1-ct1) a2,
// unp1 += ct0 a1 + ct1 a2; a1 and a2 are cleared for the next subcycle
// (three stage fields for RK3: a3 with ct2, else a3 is unused)
template <typename T, bool THREE>
__global__ void __launch_bounds__(256) k_distribute(FieldPtrsW<T> a1, FieldPtrsW<T> a2, FieldPtrsW<T> a3, FieldPtrsW<T> ubn,
                                                     FieldPtrsW<T> ubp, T ct0, T ct1, T ct2, long ntot) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntot) return;
  const int c = blockIdx.y;
  const T x1 = a1.f[c][q], x2 = a2.f[c][q], x3 = THREE ? a3.f[c][q] : T(0);
  if (x1 == T(0) && x2 == T(0) && x3 == T(0)) return;
  if (THREE) {
    ubn.f[c][q] += (T(1) - ct0) * x1 + (T(1) - ct1) * x2 + (T(1) - ct2) * x3;
    ubp.f[c][q] += ct0 * x1 + ct1 * x2 + ct2 * x3;
    a3.f[c][q] = T(0);
  } else {
    ubn.f[c][q] += (T(1) - ct0) * x1 + (T(1) - ct1) * x2;
    ubp.f[c][q] += ct0 * x1 + ct1 * x2;
  }
  a1.f[c][q] = T(0);
  a2.f[c][q] = T(0);
}


// ---------------------------------------------------------------------------------------
// Tangent-linear form of one backward SL subcycle: with the velocity levels perturbed along
// D (dun, dunp1) and the previous map along dfo, the first-order change of the new map at the
// interior nodes (ghosts by k_periodic_ghosts).  Same recomputed stages, brackets and clamped
// fractions as the forward kernel and k_sl_adjoint, so that for every direction d the
// tangent's dJ equals the adjoint's <dJ/du, d> to rounding.
// ---------------------------------------------------------------------------------------
template <typename T, int INTEG, bool F = false>
__global__ void __launch_bounds__(256) k_sl_tangent(DevGrid<T> g, VelFields<T> V, VelFields<T> D, FieldPtrs<T> fmo, FieldPtrs<T> dfo,
                                                     FieldPtrsW<T> dfn, StageTimes S, T dt, int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const T HALF = T(1) / T(2);
  const int no[3] = {i, j, k};
  const T x0[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  const T ct0 = T(S.ct[0]), omc0 = T(1) - ct0;
  T u1[3], du1[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    u1[c] = omc0 * __ldg(V.un[c] + p) + ct0 * __ldg(V.unp1[c] + p);
    du1[c] = omc0 * __ldg(D.un[c] + p) + ct0 * __ldg(D.unp1[c] + p);
  }
  T x[3], dx[3];
  // one LINEAR stage sample at xs (moved by dxs) of V (value) and of the direction D (tangent)
  auto stage_tan = [&](const T xs[3], const T dxs[3], T omc, T ct, T u[3], T du[3]) {
    LinStencilAD<T> st;
    lin_stencil_ad(g, xs, no, st);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      u[c] = lin_apply_blend<T, T>(st.st, V.un[c], V.unp1[c], omc, ct);
      du[c] = lin_apply_blend<T, T>(st.st, D.un[c], D.unp1[c], omc, ct);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int cq = corner(st.st, q);
      T dwq = T(0);
#pragma unroll
      for (int d = 0; d < 3; d++) dwq += dweight(st.t, q, d) * st.dtdx[d] * dxs[d];
#pragma unroll
      for (int c = 0; c < 3; c++) du[c] += dwq * (omc * __ldg(V.un[c] + cq) + ct * __ldg(V.unp1[c] + cq));
    }
  };
  if (INTEG == RK4) {
    const T R4_HALF = T(1) / T(2), R4_SIXTH = T(1) / T(6), R4_THIRD = T(1) / T(3);
    const T r1 = T(S.ct[1]), q1 = T(1) - r1, r2 = T(S.ct[2]), q2 = T(1) - r2, r3 = T(S.ct[3]), q3 = T(1) - r3;
    T kk[3], dk[3], acc[3], dacc[3], xs[3], dxs[3], u[3], du[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u1[c];
      dk[c] = dt * du1[c];
      acc[c] = x0[c] + R4_SIXTH * kk[c];
      dacc[c] = R4_SIXTH * dk[c];
      xs[c] = x0[c] + R4_HALF * kk[c];
      dxs[c] = R4_HALF * dk[c];
    }
    stage_tan(xs, dxs, q1, r1, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      dk[c] = dt * du[c];
      acc[c] = acc[c] + R4_THIRD * kk[c];
      dacc[c] = dacc[c] + R4_THIRD * dk[c];
      xs[c] = x0[c] + R4_HALF * kk[c];
      dxs[c] = R4_HALF * dk[c];
    }
    stage_tan(xs, dxs, q2, r2, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      dk[c] = dt * du[c];
      acc[c] = acc[c] + R4_THIRD * kk[c];
      dacc[c] = dacc[c] + R4_THIRD * dk[c];
      xs[c] = x0[c] + kk[c];
      dxs[c] = dk[c];
    }
    stage_tan(xs, dxs, q3, r3, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      x[c] = acc[c] + R4_SIXTH * kk[c];
      dx[c] = dacc[c] + R4_SIXTH * (dt * du[c]);
    }
  } else if (INTEG == RK3) {
    const T SIXTH = T(1) / T(6), TWOTHIRD = T(2) / T(3), TWO = T(2);
    const T ct1 = T(S.ct[1]), omc1 = T(1) - ct1, ct2 = T(S.ct[2]), omc2 = T(1) - ct2;
    T k[3], dk[3], acc[3], dacc[3], xs[3], dxs[3], u[3], du[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u1[c];
      dk[c] = dt * du1[c];
      acc[c] = x0[c] + SIXTH * k[c];
      dacc[c] = SIXTH * dk[c];
      xs[c] = x0[c] + HALF * k[c];
      dxs[c] = HALF * dk[c];
    }
    stage_tan(xs, dxs, omc1, ct1, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      dk[c] = dt * du[c];
      xs[c] = x0[c] + TWO * k[c];
      dxs[c] = TWO * dk[c];
      acc[c] = acc[c] + TWOTHIRD * k[c];
      dacc[c] = dacc[c] + TWOTHIRD * dk[c];
    }
    stage_tan(xs, dxs, omc2, ct2, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * k[c];
      dx[c] = dacc[c] + SIXTH * (dt * du[c]);
    }
  } else if (INTEG == RK2) {
    const T ct1 = T(S.ct[1]), omc1 = T(1) - ct1;
    T xh[3], dxh[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      xh[c] = x0[c] + HALF * dt * u1[c];
      dxh[c] = HALF * dt * du1[c];
    }
    LinStencilAD<T> s2;
    lin_stencil_ad(g, xh, no, s2);
    T u2[3], du2[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      u2[c] = lin_apply_blend<T, T>(s2.st, V.un[c], V.unp1[c], omc1, ct1);
      du2[c] = lin_apply_blend<T, T>(s2.st, D.un[c], D.unp1[c], omc1, ct1);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int cq = corner(s2.st, q);
      T dwq = T(0);
#pragma unroll
      for (int d = 0; d < 3; d++) dwq += dweight(s2.t, q, d) * s2.dtdx[d] * dxh[d];
#pragma unroll
      for (int c = 0; c < 3; c++) du2[c] += dwq * (omc1 * __ldg(V.un[c] + cq) + ct1 * __ldg(V.unp1[c] + cq));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x0[c] + dt * u2[c];
      dx[c] = dt * du2[c];
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x0[c] + dt * u1[c];
      dx[c] = dt * du1[c];
    }
  }
  // the forward kernel's plane projection and particle boundary condition, and their tangents
  {
    int nb[3] = {i, j, k};
    project_plane(g, nb, x);
    const int sa = g.P.single_axis;
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (c == sa) dx[c] = T(0);
    bool proj = false;
    T bn[3];
    if (F && bc_record(g, nb, x, proj, bn)) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        x[c] = x0[c];
        dx[c] = T(0);
      }
    } else if (proj) {
      const T d = dx[0] * bn[0] + dx[1] * bn[1] + dx[2] * bn[2];
#pragma unroll
      for (int c = 0; c < 3; c++) dx[c] -= bn[c] * d;
    }
  }
  LinStencilAD<T> s3;
  lin_stencil_ad(g, x, no, s3);
  // fm_new = fm_old(x) + (x - x0)
  T out[3] = {dx[0], dx[1], dx[2]};
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int cq = corner(s3.st, q);
    const T wq = s3.st.w[q];
    T dwq = T(0);
#pragma unroll
    for (int d = 0; d < 3; d++) dwq += dweight(s3.t, q, d) * s3.dtdx[d] * dx[d];
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] += wq * __ldg(dfo.f[c] + cq) + dwq * __ldg(fmo.f[c] + cq);
  }
  // the mask factor and the flow-map boundary rule (the forward kernel's vpre / vfin)
  const int fl = F ? (int)g.flag[p] : (int)LCS_INTERNAL;
  const T mask = fl != LCS_MASK ? T(1) : T(0);
  const bool zero = F && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
  T vpre[3], vfin[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    vpre[c] = out[c] * mask;
    vfin[c] = zero ? T(0) : vpre[c];
    dfn.f[c][p] = vfin[c];
  }
  if (F) write_ghosts<T, true, GHOST_FM>(g, dfn.f, i, j, k, vpre, vfin, err);
}

// ---------------------------------------------------------------------------------------
// CUBIC interpolation (the not-a-knot cubic B-spline on every axis, the library's SPLINE4
// kernels): basis values exactly as basis_values<T, 4, false> forms them (spline.cuh, the
// Cox-de Boor recurrence with the interval's reciprocal spans), so the recomputed stage
// positions are the forward kernel's, and the derivative of each cubic basis function from the
// quadratic ones of the same recurrence: B'(i,4) = 3 (B(i,3) / (t(i+3) - t(i)) - B(i+1,3) /
// (t(i+4) - t(i+1))), whose reciprocal spans are the recurrence's third-level slots.
// ---------------------------------------------------------------------------------------
template <typename T>
struct CubicStencil {
  int p0;       // padded index of the first coefficient
  T b[3][4];    // basis values per axis
  T db[3][4];   // their derivatives in the coordinate
};

template <typename T>
__device__ __forceinline__ void cubic_basis_d(const SplineAxis<T> &A, int l, T x, T *b, T *db) {
  const T *r = A.rinv + (size_t)(l - 1) * 6;
  T dr[4], dl[4], b3[3] = {T(0), T(0), T(0)};
  b[0] = T(1);
  int slot = 0;
#pragma unroll
  for (int j = 1; j < 4; j++) {
    dr[j] = __ldg(A.t + l + j - 1) - x;
    dl[j] = x - __ldg(A.t + l - j);
    T prev = T(0);
#pragma unroll
    for (int m = 1; m <= 3; m++) {
      if (m > j) break;
      const T vm = b[m - 1] * __ldg(r + slot++);
      b[m - 1] = vm * dr[m] + prev;
      prev = vm * dl[j + 1 - m];
    }
    b[j] = prev;
    if (j == 2) {
      b3[0] = b[0];
      b3[1] = b[1];
      b3[2] = b[2];
    }
  }
  const T R0 = __ldg(r + 3), R1 = __ldg(r + 4), R2 = __ldg(r + 5);
  db[0] = T(-3) * (b3[0] * R0);
  db[1] = T(3) * (b3[0] * R0 - b3[1] * R1);
  db[2] = T(3) * (b3[1] * R1 - b3[2] * R2);
  db[3] = T(3) * (b3[2] * R2);
}

// spline_stencil<T, 4, false> with the derivatives; false where db3val returns 0
template <typename T>
__device__ __forceinline__ bool cubic_stencil_d(const DevGrid<T> &g, const SplineAxes<T> &S, const T x[3], const int no[3], CubicStencil<T> &st) {
  int c0[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const SplineAxis<T> &A = S.ax[a];
    const int n = A.n, k = 4;
    const T tfirst = __ldg(A.t), tlast = __ldg(A.t + n + k - 1);
    if (!(x[a] >= tfirst) || x[a] > tlast) return false;
    int l;
    if (a == 0) {
      l = (x[a] >= __ldg(A.t + n)) ? n : knot_interval(A.t, x[a], k, n, no[a] + k - 1);
    } else {
      if (x[a] >= tlast) return false;
      l = knot_interval(A.t, x[a], k, n, no[a] + k - 1);
    }
    cubic_basis_d(A, l, x[a], st.b[a], st.db[a]);
    c0[a] = l - k;
  }
  st.p0 = pidx(g.P.sx, g.P.sxy, c0[0], c0[1], c0[2]);
  return true;
}

// value (spline_contract's order) and gradient of one component; tap(q) the coefficient at
// padded index q
template <typename T, typename Tap>
__device__ __forceinline__ T cubic_value_grad(const DevGrid<T> &g, const CubicStencil<T> &st, Tap tap, T gr[3]) {
  T vz = T(0), gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
  for (int c2 = 0; c2 < 4; c2++) {
    T vy = T(0), vyx = T(0), vyy = T(0);
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) {
      T vx = T(0), dx = T(0);
#pragma unroll
      for (int c0 = 0; c0 < 4; c0++) {
        const T q = tap(st.p0 + c0 + c1 * g.P.sx + c2 * g.P.sxy);
        vx += st.b[0][c0] * q;
        dx += st.db[0][c0] * q;
      }
      vy += st.b[1][c1] * vx;
      vyx += st.b[1][c1] * dx;
      vyy += st.db[1][c1] * vx;
    }
    vz += st.b[2][c2] * vy;
    gx += st.b[2][c2] * vyx;
    gy += st.b[2][c2] * vyy;
    gz += st.db[2][c2] * vy;
  }
  gr[0] = gx;
  gr[1] = gy;
  gr[2] = gz;
  return vz;
}

// adjoint of the contraction: coefficient q gets its basis product times a[c] (component c)
template <typename T>
__device__ __forceinline__ void cubic_scatter(const DevGrid<T> &g, const CubicStencil<T> &st, FieldPtrsW<T> C, const T a[3]) {
#pragma unroll
  for (int c2 = 0; c2 < 4; c2++)
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) {
      const T w21 = st.b[2][c2] * st.b[1][c1];
#pragma unroll
      for (int c0 = 0; c0 < 4; c0++) {
        const T w = w21 * st.b[0][c0];
        const int q = st.p0 + c0 + c1 * g.P.sx + c2 * g.P.sxy;
#pragma unroll
        for (int c = 0; c < 3; c++)
          if (a[c] != T(0)) atomicAdd(C.f[c] + q, w * a[c]);
      }
    }
}

// One sampled stage of the cubic sweeps: the blended velocity (1-ct) cn + ct cp at xs (the
// coefficients of the two levels blended tap by tap as k_blend blends them) and its gradient.
template <typename T>
struct CubicSample {
  CubicStencil<T> st;
  bool ok;
  T u[3], gr[3][3];  // gr[c][d] = d u_c / d x_d
};

template <typename T>
__device__ __forceinline__ void cubic_sample(const DevGrid<T> &g, const SplineAxes<T> &sa, FieldPtrs<T> cn, FieldPtrs<T> cp, T omc, T ct,
                                             const T xs[3], const int no[3], CubicSample<T> &s) {
  s.ok = cubic_stencil_d(g, sa, xs, no, s.st);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (!s.ok) {
      s.u[c] = T(0);
      s.gr[c][0] = s.gr[c][1] = s.gr[c][2] = T(0);
      continue;
    }
    const T *a = cn.f[c], *b = cp.f[c];
    s.u[c] = cubic_value_grad(g, s.st, [&](int q) { return omc * __ldg(a + q) + ct * __ldg(b + q); }, s.gr[c]);
  }
}

// ---------------------------------------------------------------------------------------
// Adjoint of one backward SL subcycle with CUBIC interpolation (k_sl_subcycle<..., SPLINE4>,
// no flags): the forward stages recomputed from the coefficient levels cn, cp and the previous
// map's coefficients cfm; the previous map's adjoint goes to cbo in coefficient space (the
// transposed fit follows on the host side), the off-node stages' velocity adjoints to a2, a3 in
// coefficient space, the node stage's to a1 in value space.
// ---------------------------------------------------------------------------------------
template <typename T, int INTEG>
__global__ void __launch_bounds__(128) k_sl_adjoint_cubic(DevGrid<T> g, SplineAxes<T> sa, VelFields<T> V, FieldPtrs<T> cn, FieldPtrs<T> cp,
                                                           FieldPtrs<T> cfm, FieldPtrs<T> fbn, FieldPtrsW<T> cbo, FieldPtrsW<T> a1,
                                                           FieldPtrsW<T> a2, FieldPtrsW<T> a3, StageTimes S, T dt) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const T a[3] = {fbn.f[0][p], fbn.f[1][p], fbn.f[2][p]};
  if (a[0] == T(0) && a[1] == T(0) && a[2] == T(0)) return;
  const T HALF = T(1) / T(2), SIXTH = T(1) / T(6), TWOTHIRD = T(2) / T(3), TWO = T(2);
  const int no[3] = {i, j, k};
  const T x0[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  const T ct0 = T(S.ct[0]), omc0 = T(1) - ct0;
  const T ct1 = T(S.ct[1]), omc1 = T(1) - ct1, ct2 = T(S.ct[2]), omc2 = T(1) - ct2;
  T u1[3];
#pragma unroll
  for (int c = 0; c < 3; c++) u1[c] = omc0 * __ldg(V.un[c] + p) + ct0 * __ldg(V.unp1[c] + p);
  // --- forward recomputation (integrate<>, first stage on the node) ---
  CubicSample<T> s2, s3, s4;
  T x[3];
  if (INTEG == RK4) {
    const T ct3 = T(S.ct[3]), omc3 = T(1) - ct3, THIRD = T(1) / T(3);
    T kk[3], acc[3], xs[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u1[c];
      acc[c] = x0[c] + SIXTH * kk[c];
      xs[c] = x0[c] + HALF * kk[c];
    }
    cubic_sample(g, sa, cn, cp, omc1, ct1, xs, no, s2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * s2.u[c];
      acc[c] = acc[c] + THIRD * kk[c];
      xs[c] = x0[c] + HALF * kk[c];
    }
    cubic_sample(g, sa, cn, cp, omc2, ct2, xs, no, s3);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * s3.u[c];
      acc[c] = acc[c] + THIRD * kk[c];
      xs[c] = x0[c] + kk[c];
    }
    cubic_sample(g, sa, cn, cp, omc3, ct3, xs, no, s4);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * s4.u[c];
      x[c] = acc[c] + SIXTH * kk[c];
    }
  } else if (INTEG == RK3) {
    T kk[3], acc[3], xs[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u1[c];
      acc[c] = x0[c] + SIXTH * kk[c];
      xs[c] = x0[c] + HALF * kk[c];
    }
    cubic_sample(g, sa, cn, cp, omc1, ct1, xs, no, s2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * s2.u[c];
      xs[c] = x0[c] + TWO * kk[c];
      acc[c] = acc[c] + TWOTHIRD * kk[c];
    }
    cubic_sample(g, sa, cn, cp, omc2, ct2, xs, no, s3);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * s3.u[c];
      x[c] = acc[c] + SIXTH * kk[c];
    }
  } else if (INTEG == RK2) {
    T xs[3];
#pragma unroll
    for (int c = 0; c < 3; c++) xs[c] = x0[c] + HALF * dt * u1[c];
    cubic_sample(g, sa, cn, cp, omc1, ct1, xs, no, s2);
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = x0[c] + dt * s2.u[c];
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = x0[c] + dt * u1[c];
  }
  // --- fm_new = fm_old(x) + (x - x0) ---
  T xb[3] = {a[0], a[1], a[2]};
  {
    CubicStencil<T> sf;
    if (cubic_stencil_d(g, sa, x, no, sf)) {
      cubic_scatter(g, sf, cbo, a);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        T gr[3];
        const T *f = cfm.f[c];
        (void)cubic_value_grad(g, sf, [&](int q) { return __ldg(f + q); }, gr);
#pragma unroll
        for (int d = 0; d < 3; d++) xb[d] += a[c] * gr[d];
      }
    }
  }
  // --- stages: a sampled stage's velocity adjoint ub into coefficient space (as = a2 or a3),
  // returning the adjoint of the sample position ---
  auto stage_back = [&](const CubicSample<T> &sm, const T ub[3], FieldPtrsW<T> as, T pb[3]) {
    pb[0] = pb[1] = pb[2] = T(0);
    if (!sm.ok) return;
    cubic_scatter(g, sm.st, as, ub);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int d = 0; d < 3; d++) pb[d] += ub[c] * sm.gr[c][d];
  };
  T u1b[3];
  if (INTEG == RK4) {
    // the two half-step stages share ct and go to a2, the last stage to a3 (with ct[3])
    const T THIRD = T(1) / T(3);
    T k3b[3], k2b[3], k1b[3], ub[3], pb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k1b[c] = SIXTH * xb[c];
      k2b[c] = THIRD * xb[c];
      k3b[c] = THIRD * xb[c];
      ub[c] = dt * (SIXTH * xb[c]);
    }
    stage_back(s4, ub, a3, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k3b[c] += pb[c];
      ub[c] = dt * k3b[c];
    }
    stage_back(s3, ub, a2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k2b[c] += HALF * pb[c];
      ub[c] = dt * k2b[c];
    }
    stage_back(s2, ub, a2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * (k1b[c] + HALF * pb[c]);
  } else if (INTEG == RK3) {
    T k2b[3], k1b[3], ub[3], pb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k2b[c] = TWOTHIRD * xb[c];
      k1b[c] = SIXTH * xb[c];
      ub[c] = dt * (SIXTH * xb[c]);
    }
    stage_back(s3, ub, a3, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      k2b[c] += TWO * pb[c];
      ub[c] = dt * k2b[c];
    }
    stage_back(s2, ub, a2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * (k1b[c] + HALF * pb[c]);
  } else if (INTEG == RK2) {
    T ub[3], pb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) ub[c] = dt * xb[c];
    stage_back(s2, ub, a2, pb);
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = HALF * dt * pb[c];
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) u1b[c] = dt * xb[c];
  }
#pragma unroll
  for (int c = 0; c < 3; c++) a1.f[c][p] = u1b[c];
}

// Tangent-linear form of the CUBIC subcycle: direction levels D (values, for the node stage) and
// dcn, dcp (their coefficients), the previous map's tangent coefficients dcfm.
template <typename T, int INTEG>
__global__ void __launch_bounds__(128) k_sl_tangent_cubic(DevGrid<T> g, SplineAxes<T> sa, VelFields<T> V, VelFields<T> D, FieldPtrs<T> cn,
                                                           FieldPtrs<T> cp, FieldPtrs<T> dcn, FieldPtrs<T> dcp, FieldPtrs<T> cfm,
                                                           FieldPtrs<T> dcfm, FieldPtrsW<T> dfn, StageTimes S, T dt) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const T HALF = T(1) / T(2), SIXTH = T(1) / T(6), TWOTHIRD = T(2) / T(3), TWO = T(2);
  const int no[3] = {i, j, k};
  const T x0[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  const T ct0 = T(S.ct[0]), omc0 = T(1) - ct0;
  const T ct1 = T(S.ct[1]), omc1 = T(1) - ct1, ct2 = T(S.ct[2]), omc2 = T(1) - ct2;
  T u1[3], du1[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    u1[c] = omc0 * __ldg(V.un[c] + p) + ct0 * __ldg(V.unp1[c] + p);
    du1[c] = omc0 * __ldg(D.un[c] + p) + ct0 * __ldg(D.unp1[c] + p);
  }
  // velocity at xs and its first-order change for a move dxs of the point
  auto stage_tan = [&](const T xs[3], const T dxs[3], T omc, T ct, T u[3], T du[3]) {
    CubicSample<T> sm;
    cubic_sample(g, sa, cn, cp, omc, ct, xs, no, sm);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      u[c] = sm.u[c];
      du[c] = T(0);
      if (!sm.ok) continue;
      T gr[3];
      const T *a = dcn.f[c], *b = dcp.f[c];
      du[c] = cubic_value_grad(g, sm.st, [&](int q) { return omc * __ldg(a + q) + ct * __ldg(b + q); }, gr);
#pragma unroll
      for (int d = 0; d < 3; d++) du[c] += sm.gr[c][d] * dxs[d];
    }
  };
  T x[3], dx[3];
  if (INTEG == RK4) {
    const T R4_HALF = T(1) / T(2), R4_SIXTH = T(1) / T(6), R4_THIRD = T(1) / T(3);
    const T r1 = T(S.ct[1]), q1 = T(1) - r1, r2 = T(S.ct[2]), q2 = T(1) - r2, r3 = T(S.ct[3]), q3 = T(1) - r3;
    T kk[3], dk[3], acc[3], dacc[3], xs[3], dxs[3], u[3], du[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u1[c];
      dk[c] = dt * du1[c];
      acc[c] = x0[c] + R4_SIXTH * kk[c];
      dacc[c] = R4_SIXTH * dk[c];
      xs[c] = x0[c] + R4_HALF * kk[c];
      dxs[c] = R4_HALF * dk[c];
    }
    stage_tan(xs, dxs, q1, r1, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      dk[c] = dt * du[c];
      acc[c] = acc[c] + R4_THIRD * kk[c];
      dacc[c] = dacc[c] + R4_THIRD * dk[c];
      xs[c] = x0[c] + R4_HALF * kk[c];
      dxs[c] = R4_HALF * dk[c];
    }
    stage_tan(xs, dxs, q2, r2, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      dk[c] = dt * du[c];
      acc[c] = acc[c] + R4_THIRD * kk[c];
      dacc[c] = dacc[c] + R4_THIRD * dk[c];
      xs[c] = x0[c] + kk[c];
      dxs[c] = dk[c];
    }
    stage_tan(xs, dxs, q3, r3, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      x[c] = acc[c] + R4_SIXTH * kk[c];
      dx[c] = dacc[c] + R4_SIXTH * (dt * du[c]);
    }
  } else if (INTEG == RK3) {
    T kk[3], dk[3], acc[3], dacc[3], xs[3], dxs[3], u[3], du[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u1[c];
      dk[c] = dt * du1[c];
      acc[c] = x0[c] + SIXTH * kk[c];
      dacc[c] = SIXTH * dk[c];
      xs[c] = x0[c] + HALF * kk[c];
      dxs[c] = HALF * dk[c];
    }
    stage_tan(xs, dxs, omc1, ct1, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      dk[c] = dt * du[c];
      xs[c] = x0[c] + TWO * kk[c];
      dxs[c] = TWO * dk[c];
      acc[c] = acc[c] + TWOTHIRD * kk[c];
      dacc[c] = dacc[c] + TWOTHIRD * dk[c];
    }
    stage_tan(xs, dxs, omc2, ct2, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * kk[c];
      dx[c] = dacc[c] + SIXTH * (dt * du[c]);
    }
  } else if (INTEG == RK2) {
    T xs[3], dxs[3], u[3], du[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      xs[c] = x0[c] + HALF * dt * u1[c];
      dxs[c] = HALF * dt * du1[c];
    }
    stage_tan(xs, dxs, omc1, ct1, u, du);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x0[c] + dt * u[c];
      dx[c] = dt * du[c];
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x0[c] + dt * u1[c];
      dx[c] = dt * du1[c];
    }
  }
  // fm_new = fm_old(x) + (x - x0)
  T out[3] = {dx[0], dx[1], dx[2]};
  CubicStencil<T> sf;
  if (cubic_stencil_d(g, sa, x, no, sf)) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      T gr[3], g2[3];
      const T *f = cfm.f[c], *df = dcfm.f[c];
      (void)cubic_value_grad(g, sf, [&](int q) { return __ldg(f + q); }, gr);
      out[c] += cubic_value_grad(g, sf, [&](int q) { return __ldg(df + q); }, g2);
#pragma unroll
      for (int d = 0; d < 3; d++) out[c] += gr[d] * dx[d];
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) dfn.f[c][p] = out[c];
}

// Adjoint of one B-spline fit pass (k_fit_xlines / k_fit_lines): the transposed banded solves of
// spline_pull_table_transposed along every line of one axis, in place.  Line L starts at
// (L % nfast) * ls + (L / nfast) * so, its n elements es apart.
template <typename T>
__global__ void __launch_bounds__(256) k_fit_transpose(const T *__restrict__ pt, int n, FieldPtrsW<T> f, int nfast, long nlines, long ls,
                                                        long so, long es) {
  const long L = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlines) return;
  T *d = f.f[blockIdx.y] + (L % nfast) * ls + (L / nfast) * so;
  T w[3] = {T(0), T(0), T(0)};
  for (int r = 0; r < n; r++) {
    const T *c = pt + 8 * (size_t)r;
    T v = d[(long)r * es];
    v = v - w[0] * __ldg(c + 0) - w[1] * __ldg(c + 1) - w[2] * __ldg(c + 2);
    v = v * __ldg(c + 6);
    w[2] = w[1];
    w[1] = w[0];
    w[0] = v;
    d[(long)r * es] = v;
  }
  w[0] = w[1] = w[2] = T(0);
  for (int r = n - 1; r >= 0; r--) {
    const T *c = pt + 8 * (size_t)r;
    T v = d[(long)r * es];
    v = v - w[0] * __ldg(c + 3) - w[1] * __ldg(c + 4) - w[2] * __ldg(c + 5);
    w[2] = w[1];
    w[1] = w[0];
    w[0] = v;
    d[(long)r * es] = v;
  }
}

// velocity adjoint of one CUBIC subcycle onto the two levels: the node stage (a1, values) into
// ubn / ubp with (1-ct0, ct0), the off-node stages (a2 with ct1, a3 with ct2; coefficients)
// into cbn / cbp; the stage fields are cleared for the next subcycle
template <typename T, bool THREE>
__global__ void __launch_bounds__(256) k_distribute_cubic(FieldPtrsW<T> a1, FieldPtrsW<T> a2, FieldPtrsW<T> a3, FieldPtrsW<T> ubn,
                                                           FieldPtrsW<T> ubp, FieldPtrsW<T> cbn, FieldPtrsW<T> cbp, T ct0, T ct1, T ct2,
                                                           long ntot) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntot) return;
  const int c = blockIdx.y;
  const T x1 = a1.f[c][q], x2 = a2.f[c][q], x3 = THREE ? a3.f[c][q] : T(0);
  if (x1 != T(0)) {
    ubn.f[c][q] += (T(1) - ct0) * x1;
    ubp.f[c][q] += ct0 * x1;
    a1.f[c][q] = T(0);
  }
  if (x2 != T(0) || x3 != T(0)) {
    cbn.f[c][q] += (T(1) - ct1) * x2 + (T(1) - ct2) * x3;
    cbp.f[c][q] += ct1 * x2 + ct2 * x3;
    a2.f[c][q] = T(0);
    if (THREE) a3.f[c][q] = T(0);
  }
}

// dst += src (three components, padded)
template <typename T>
__global__ void __launch_bounds__(256) k_add3(FieldPtrsW<T> dst, FieldPtrs<T> src, long ntot) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntot) return;
  const int c = blockIdx.y;
  dst.f[c][q] += src.f[c][q];
}

// source interior index of a padded cell along one periodic axis
__device__ __forceinline__ int wrap_index(int v, int n) { return v < 1 ? v + n : (v > n ? v - n : v); }

// Adjoint of the periodic ghost fill (write_ghosts rule 0 on every face, edge and corner):
// each ghost's adjoint is added to its source node and cleared.
template <typename T>
__global__ void __launch_bounds__(256) k_fold_ghosts(DevGrid<T> g, FieldPtrsW<T> f, long ntot) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntot) return;
  const int i = (int)(p % g.P.sx), j = (int)((p / g.P.sx) % (g.P.sxy / g.P.sx)), k = (int)(p / g.P.sxy);
  const int si = wrap_index(i, g.P.n[0]), sj = wrap_index(j, g.P.n[1]), sk = wrap_index(k, g.P.n[2]);
  if (si == i && sj == j && sk == k) return;
  const int q = pidx(g.P.sx, g.P.sxy, si, sj, sk);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const T v = f.f[c][p];
    if (v != T(0)) atomicAdd(f.f[c] + q, v);
    f.f[c][p] = T(0);
  }
}

// periodic ghost fill of a tangent map (write_ghosts rule 0 on every face, edge and corner;
// the transpose of k_fold_ghosts)
template <typename T>
__global__ void __launch_bounds__(256) k_periodic_ghosts(DevGrid<T> g, FieldPtrsW<T> f, long ntot) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntot) return;
  const int i = (int)(p % g.P.sx), j = (int)((p / g.P.sx) % (g.P.sxy / g.P.sx)), k = (int)(p / g.P.sxy);
  const int si = wrap_index(i, g.P.n[0]), sj = wrap_index(j, g.P.n[1]), sk = wrap_index(k, g.P.n[2]);
  if (si == i && sj == j && sk == k) return;
  const int q = pidx(g.P.sx, g.P.sxy, si, sj, sk);
#pragma unroll
  for (int c = 0; c < 3; c++) f.f[c][p] = f.f[c][q];
}

// ---------------------------------------------------------------------------------------
// Boundary flags (walls, slip, inflow / outflow, masks, 2-D).  The forward ghost fill
// (write_ghosts, device_common.cuh) gives every ghost cell one rule: 0 the periodic image of a
// node's value before the interior zeroing (vpre), 1 zero, 2 a copy of its nearest node's final
// value (vfin); the interior zeroing is: flow map at MASK / INFLOW / OUTFLOW nodes, velocity at
// MASK nodes, and the flow map's pre-zeroing value carries the mask factor (0 at MASK nodes).
// Its adjoint runs in three passes over a padded adjoint field: copy ghosts into their nodes,
// clear the nodes whose final value is zero, image ghosts into their nodes (times the mask for
// the flow map) -- leaving at each node the adjoint of the quantity the subcycle computes before
// any zeroing.
// ---------------------------------------------------------------------------------------
template <typename T, int KIND>
__global__ void __launch_bounds__(256) k_fold_copy(DevGrid<T> g, FieldPtrsW<T> f, long ntot) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntot) return;
  const int i = (int)(p % g.P.sx), j = (int)((p / g.P.sx) % (g.P.sxy / g.P.sx)), k = (int)(p / g.P.sxy);
  if (i >= 1 && j >= 1 && k >= 1 && i <= g.P.n[0] && j <= g.P.n[1] && k <= g.P.n[2]) return;
  const int rule = ghost_rule(KIND, (int)g.flag[p]);
  if (rule == 0) return;
  if (rule == 2) {
    const int q = pidx(g.P.sx, g.P.sxy, min(max(i, 1), g.P.n[0]), min(max(j, 1), g.P.n[1]), min(max(k, 1), g.P.n[2]));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T v = f.f[c][p];
      if (v != T(0)) atomicAdd(f.f[c] + q, v);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) f.f[c][p] = T(0);
}

template <typename T, int KIND>
__global__ void __launch_bounds__(256) k_fold_zero(DevGrid<T> g, FieldPtrsW<T> f) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const int fl = (int)g.flag[p];
  const bool zero = KIND == GHOST_FM ? (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW) : fl == LCS_MASK;
  if (!zero) return;
#pragma unroll
  for (int c = 0; c < 3; c++) f.f[c][p] = T(0);
}

template <typename T, int KIND>
__global__ void __launch_bounds__(256) k_fold_image(DevGrid<T> g, FieldPtrsW<T> f, long ntot) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntot) return;
  const int i = (int)(p % g.P.sx), j = (int)((p / g.P.sx) % (g.P.sxy / g.P.sx)), k = (int)(p / g.P.sxy);
  if (i >= 1 && j >= 1 && k >= 1 && i <= g.P.n[0] && j <= g.P.n[1] && k <= g.P.n[2]) return;
  if (ghost_rule(KIND, (int)g.flag[p]) != 0) return;  // cleared by k_fold_copy
  const int q = pidx(g.P.sx, g.P.sxy, wrap_index(i, g.P.n[0]), wrap_index(j, g.P.n[1]), wrap_index(k, g.P.n[2]));
  const T m = (KIND == GHOST_FM && g.flag[q] == LCS_MASK) ? T(0) : T(1);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const T v = f.f[c][p];
    if (v != T(0)) atomicAdd(f.f[c] + q, m * v);
    f.f[c][p] = T(0);
  }
}

// interior of a padded field -> compact i-fastest arrays (the composed map of an h = T frame)
template <typename T>
__global__ void __launch_bounds__(256) k_interior(DevGrid<T> g, FieldPtrs<T> src, FieldPtrsW<T> dst) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k), q = interior_index(g.P.n, i, j, k);
#pragma unroll
  for (int c = 0; c < 3; c++) dst.f[c][q] = src.f[c][p];
}

// The FTLE at node (i, j, k) linearised in the flow map: the central-difference gradient G,
// the neighbours and spacings it used, the largest eigenvalue lam of G^T G and its unit
// eigenvector v.  False where the derivative is zero (FTLE at its tiny floor) or undefined
// (repeated largest eigenvalue).
template <typename T>
struct FtleLin {
  double G[3][3], den[3], v[3], Gv[3], lam;
  int qp[3], qm[3];
};

template <typename T>
__device__ __forceinline__ bool ftle_linearise(const DevGrid<T> &g, const FieldPtrs<T> &fm, int i, int j, int k, FtleLin<T> &L) {
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (g.P.n[a] == 1) {
      for (int c = 0; c < 3; c++) L.G[c][a] = 0.0;
      L.den[a] = 0.0;
      L.qp[a] = L.qm[a] = -1;
      continue;
    }
    // the neighbour value k_ftle's fm_neighbour reads: the node in range, its periodic image, the
    // node itself behind a copy (rule 2) ghost, zero behind any other ghost (-1)
    auto nbr = [&](int step) -> int {
      int q[3] = {i, j, k};
      q[a] = idx[a] + step;
      if (q[a] >= 1 && q[a] <= g.P.n[a]) return pidx(g.P.sx, g.P.sxy, q[0], q[1], q[2]);
      if (g.P.per[a]) {
        q[a] = wrap_index(q[a], g.P.n[a]);
        return pidx(g.P.sx, g.P.sxy, q[0], q[1], q[2]);
      }
      if (g.P.has_flags && ghost_rule(GHOST_FM, (int)g.flag[pidx(g.P.sx, g.P.sxy, q[0], q[1], q[2])]) == 2)
        return pidx(g.P.sx, g.P.sxy, i, j, k);
      return -1;
    };
    L.qp[a] = nbr(+1);
    L.qm[a] = nbr(-1);
    L.den[a] = (double)(__ldg(g.lt[a] + idx[a] + 1) - __ldg(g.lt[a] + idx[a] - 1));
    for (int c = 0; c < 3; c++) {
      const T fp = L.qp[a] >= 0 ? fm.f[c][L.qp[a]] : T(0), fq = L.qm[a] >= 0 ? fm.f[c][L.qm[a]] : T(0);
      L.G[c][a] = (double)(fp - fq) / L.den[a];
    }
  }
  double C[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) C[a][b] = L.G[0][a] * L.G[0][b] + L.G[1][a] * L.G[1][b] + L.G[2][a] * L.G[2][b];
  const double lam = eig3_max_closed(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
  const double tiny = sizeof(T) == 8 ? DBL_MIN : (double)FLT_MIN;
  if (!(sqrt(lam) > tiny)) return false;  // max(sqrt(W3), tiny) is constant there
  // unit eigenvector of lam: the largest cross product of two rows of C - lam I
  const double r[3][3] = {{C[0][0] - lam, C[0][1], C[0][2]}, {C[1][0], C[1][1] - lam, C[1][2]}, {C[2][0], C[2][1], C[2][2] - lam}};
  double best = 0.0;
  L.v[0] = L.v[1] = L.v[2] = 0.0;
  for (int m = 0; m < 3; m++) {
    const double *x = r[m], *y = r[(m + 1) % 3];
    const double cx[3] = {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    const double nn = cx[0] * cx[0] + cx[1] * cx[1] + cx[2] * cx[2];
    if (nn > best) {
      best = nn;
      L.v[0] = cx[0];
      L.v[1] = cx[1];
      L.v[2] = cx[2];
    }
  }
  if (!(best > 0.0)) return false;  // repeated largest eigenvalue: no unique derivative direction
  const double s = 1.0 / sqrt(best);
  for (int a = 0; a < 3; a++) L.v[a] *= s;
  for (int c = 0; c < 3; c++) L.Gv[c] = L.G[c][0] * L.v[0] + L.G[c][1] * L.v[1] + L.G[c][2] * L.v[2];
  L.lam = lam;
  return true;
}

// ---------------------------------------------------------------------------------------
// Adjoint of compute_ftle on a periodic grid: FTLE = log(sqrt(lambda))/T with lambda the
// largest eigenvalue of C = G^T G, G the central-difference gradient of the displacement.
// d lambda / d G = 2 (G v) v^T with v the unit eigenvector; the central differences are
// transposed onto the two neighbours (periodic images wrapped to their source nodes).
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_ftle_adjoint(DevGrid<T> g, FieldPtrs<T> fm, const T *__restrict__ wgt, T Tint, FieldPtrsW<T> fb) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const double w = (double)wgt[interior_index(g.P.n, i, j, k)];
  if (w == 0.0) return;
  FtleLin<T> L;
  if (!ftle_linearise(g, fm, i, j, k, L)) return;
  // dJ/dG = w / (2 lam T) * 2 (G v) v^T
  const double coef = w / (L.lam * (double)Tint);
  for (int a = 0; a < 3; a++) {
    if (L.den[a] == 0.0) continue;  // singleton axis: no gradient column
    for (int c = 0; c < 3; c++) {
      const double gb = coef * L.Gv[c] * L.v[a] / L.den[a];
      if (L.qp[a] >= 0) atomicAdd(fb.f[c] + L.qp[a], T(gb));
      if (L.qm[a] >= 0) atomicAdd(fb.f[c] + L.qm[a], T(-gb));
    }
  }
}

// Tangent of compute_ftle: d lambda = 2 (G v) . (dG v), so w dFTLE = w d lambda / (2 lam T)
// per node (summed on the host).
template <typename T>
__global__ void __launch_bounds__(256) k_ftle_tangent(DevGrid<T> g, FieldPtrs<T> fm, FieldPtrs<T> dfm, const T *__restrict__ wgt, T Tint,
                                                       double *out) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int q = interior_index(g.P.n, i, j, k);
  out[q] = 0.0;
  const double w = (double)wgt[q];
  if (w == 0.0) return;
  FtleLin<T> L;
  if (!ftle_linearise(g, fm, i, j, k, L)) return;
  double dlam = 0.0;
  for (int c = 0; c < 3; c++) {
    double dGv = 0.0;
    for (int a = 0; a < 3; a++) {
      if (L.den[a] == 0.0) continue;
      const T dp = L.qp[a] >= 0 ? dfm.f[c][L.qp[a]] : T(0), dq = L.qm[a] >= 0 ? dfm.f[c][L.qm[a]] : T(0);
      dGv += (double)(dp - dq) / L.den[a] * L.v[a];
    }
    dlam += 2.0 * L.Gv[c] * dGv;
  }
  out[q] = w * dlam / (2.0 * L.lam * (double)Tint);
}

// adjoint velocity (after the ghost fold) -> caller's i-fastest arrays
template <typename T>
__global__ void __launch_bounds__(256) k_grad_out(DevGrid<T> g, FieldPtrs<T> src, T *gu, T *gv, T *gw) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k), q = interior_index(g.P.n, i, j, k);
  gu[q] = src.f[0][p];
  gv[q] = src.f[1][p];
  gw[q] = src.f[2][p];
}

template <typename T>
class Adjoint {
 public:
  explicit Adjoint(const AdjointProblem &pr) : pr_(pr) {}
  ~Adjoint() {
    if (stream_) {
      cudaStreamSynchronize(stream_);
      cudaStreamDestroy(stream_);
    }
    if (red_host_) cudaFreeHost(red_host_);
  }

  bool run(double *J, std::string &msg) {
    tangent_ = pr_.du && pr_.dv && pr_.dw && pr_.dJ;
    if (!setup(msg)) return false;
    if (!forward(J, msg)) return false;
    if (pr_.gu && pr_.gv && pr_.gw && !backward(msg)) return false;
    ACK(cudaStreamSynchronize(stream_));
    DevReduce r{};
    ACK(cudaMemcpy(&r, red_dev_, sizeof(DevReduce), cudaMemcpyDeviceToHost));
    if (r.err) {
      msg = "adjoint: device error in the advection kernels";
      return false;
    }
    return true;
  }

 private:
  bool setup(std::string &msg) {
    const int *n = pr_.n;
    if (pr_.nlevels < 2) {
      msg = "adjoint: at least two velocity levels are needed";
      return false;
    }
    if (pr_.integrator < EULER || pr_.integrator > RK4) {
      msg = "adjoint: the integrator must be EULER, TRAPEZOIDAL, RK2, RK3 or RK4";
      return false;
    }
    if (pr_.interpolator != LINEAR_I && pr_.interpolator != CUBIC_I) {
      msg = "adjoint: the interpolator must be LINEAR or CUBIC";
      return false;
    }
    cubic_ = pr_.interpolator == CUBIC_I;
    if (pr_.checkpoint_every < 1 || !(pr_.cfl > 0)) {
      msg = "adjoint: checkpoint interval and CFL must be positive";
      return false;
    }
    for (int l = 1; l < pr_.nlevels; l++)
      if (!(pr_.times[l] > pr_.times[l - 1])) {
        msg = "adjoint: level times must increase";
        return false;
      }
    std::vector<int> flag((size_t)n[0] * n[1] * n[2], 0);
    if (pr_.flag) std::memcpy(flag.data(), pr_.flag, flag.size() * sizeof(int));
    if (!hg_.build(n, pr_.x, pr_.y, pr_.z, flag.data())) {
      msg = "adjoint: " + hg_.error;
      return false;
    }
    if (hg_.P.curv) {
      msg = "adjoint: the grid must be an exact tensor product of coordinate lines";
      return false;
    }
    if (cubic_) {
      for (int a = 0; a < 3; a++)
        if (n[a] > 1 && !hg_.P.per[a]) {
          msg = "adjoint: CUBIC needs every direction periodic";
          return false;
        }
      if (hg_.P.single_axis >= 0 || hg_.P.has_flags) {
        msg = "adjoint: CUBIC needs a three-dimensional grid without boundary flags";
        return false;
      }
    }
    flags_ = hg_.P.has_flags != 0;
    N_ = (long)n[0] * n[1] * n[2];
    ntot_ = hg_.ntot();
    GridParams<T> P{};  // curv = 0 and no curvilinear tables: the adjoint runs on tensor-product grids
    const GridParams<lcsdata_t> &H = hg_.P;
    for (int a = 0; a < 3; a++) {
      P.n[a] = H.n[a];
      P.per[a] = H.per[a];
      for (int s = 0; s < 2; s++)
        for (int e = 0; e < 2; e++) P.gx[a][s][e] = (T)H.gx[a][s][e];
    }
    P.sx = H.sx;
    P.sxy = H.sxy;
    P.single_axis = H.single_axis;
    P.zquirk = H.zquirk;
    for (int q = 0; q < 6; q++) P.bb[q] = (T)H.bb[q];
    for (int d = 0; d < 27; d++)
      for (int c = 0; c < 3; c++) P.ps[d][c] = (T)H.ps[d][c];
    P.has_flags = H.has_flags;
    P.maxtrack = H.maxtrack;
    dg_.P = P;
    for (int a = 0; a < 3; a++) {
      if (!(dg_.lt[a] = upload(hg_.lt[a], msg))) return false;
      if (!(dg_.li[a] = upload(hg_.li[a], msg))) return false;
      // the reciprocals of the spans the kernels form in T
      if (!(dg_.ri[a] = upload(reciprocal_spans(std::vector<T>(hg_.li[a].begin(), hg_.li[a].end())), msg))) return false;
      if (!(dg_.invd[a] = upload(hg_.invd[a], msg))) return false;
      dg_.nrm[a] = nullptr;
    }
    dg_.flag = nullptr;
    if (flags_) {
      // the padded flags and boundary normals of the grid (the library's make_dev_grid)
      int8_t *f = pool_.alloc<int8_t>(hg_.flag.size(), msg);
      if (!f) return false;
      ACK(cudaMemcpy(f, hg_.flag.data(), hg_.flag.size(), cudaMemcpyHostToDevice));
      dg_.flag = f;
      for (int a = 0; a < 3; a++) {
        std::vector<lcsdata_t> comp(hg_.ntot(), lcsdata_t(0));
        if (!hg_.bcnorm.empty())
          std::copy(hg_.bcnorm.begin() + (size_t)a * hg_.ntot(), hg_.bcnorm.begin() + (size_t)(a + 1) * hg_.ntot(), comp.begin());
        if (!(dg_.nrm[a] = upload(comp, msg))) return false;
      }
    }
    if (cubic_) {
      // the not-a-knot cubic of every axis over its padded coordinate line (the library's
      // ensure_spline), its pull table for the fits and the transposed one for their adjoint
      for (int a = 0; a < 3; a++) {
        if (n[a] < 3) {
          msg = "adjoint: CUBIC needs at least 3 points in every direction";
          return false;
        }
        SplineAxisHost<lcsdata_t> A;
        if (!A.build(hg_.li[a], 4)) {
          msg = "adjoint: bspline: singular collocation system or bad abscissae";
          return false;
        }
        SplineAxis<T> &D = sa_.ax[a];
        D.n = A.n;
        D.k = A.k;
        const std::vector<lcsdata_t> pull = spline_pull_table(A);
        if (!(D.t = upload(A.t, msg)) || !(D.rinv = upload(A.rinv, msg)) || !(D.tu = upload(A.tu, msg)) || !(D.pull = upload(pull, msg)))
          return false;
        if (!(ptr_[a] = upload(spline_pull_table_transposed(pull, A.n), msg))) return false;
      }
    }
    ACK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    ACK(cudaMallocHost(&red_host_, sizeof(DevReduce)));
    if (!(red_dev_ = pool_.alloc<DevReduce>(1, msg))) return false;
    return true;
  }

  template <typename V>
  T *upload(const std::vector<V> &h, std::string &msg) {
    std::vector<T> tmp(h.begin(), h.end());
    T *d = pool_.alloc<T>(tmp.size(), msg);
    if (!d) return nullptr;
    if (cudaMemcpy(d, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
      msg = "adjoint: upload failed";
      return nullptr;
    }
    return d;
  }

  dim3 node_grid() const { return dim3((dg_.P.n[0] + 31) / 32, (dg_.P.n[1] + 7) / 8, dg_.P.n[2]); }

  bool field3(T *f[3], std::string &msg) {
    for (int c = 0; c < 3; c++) {
      if (!(f[c] = pool_.alloc<T>(ntot_, msg))) return false;
      ACK(cudaMemsetAsync(f[c], 0, ntot_ * sizeof(T), stream_));
    }
    return true;
  }

  // `count` padded fields carved from one zeroed allocation (one cudaMalloc for all levels)
  bool slab(std::vector<T *> &out, size_t count, std::string &msg) {
    T *base = pool_.alloc<T>(count * (size_t)ntot_, msg);
    if (!base) return false;
    ACK(cudaMemsetAsync(base, 0, count * (size_t)ntot_ * sizeof(T), stream_));
    out.assign(count, nullptr);
    for (size_t q = 0; q < count; q++) out[q] = base + q * (size_t)ntot_;
    return true;
  }

  // stage time fractions as Engine::stage_times computes them
  StageTimes stage_times(lcsdata_t t0, lcsdata_t t1, lcsdata_t t, lcsdata_t dt) const {
    const lcsdata_t HALF = lcsdata_t(1) / lcsdata_t(2);
    auto ct = [&](lcsdata_t tt) -> double {
      if (t1 == t0) return 0.0;
      lcsdata_t v = (tt - t0) / (t1 - t0);
      v = std::max(std::min(v, lcsdata_t(1)), lcsdata_t(0));
      return (double)v;
    };
    StageTimes S{};
    if (pr_.integrator == EULER) S.ct[0] = ct(t);
    else if (pr_.integrator == TRAPEZOIDAL) S.ct[0] = ct(t + HALF * dt);
    else {
      S.ct[0] = ct(t);
      S.ct[1] = ct(t + HALF * dt);
      if (pr_.integrator == RK3) S.ct[2] = ct(t + dt);
      if (pr_.integrator == RK4) {
        S.ct[2] = S.ct[1];
        S.ct[3] = ct(t + dt);
      }
    }
    return S;
  }

  bool forward(double *J, std::string &msg) {
    const int L = pr_.nlevels;
    // padded levels + CFL maxima -> subcycles of every update (set_dt, src/lp_motion_m.f90:56-127)
    if (!slab(U_, (size_t)3 * L, msg)) return false;
    cmax_.assign(L, 0.0);
    for (int l = 0; l < L; l++) {
      T *f[3] = {U_[3 * l], U_[3 * l + 1], U_[3 * l + 2]};
      DevReduce init{};
      double big = std::numeric_limits<double>::max();
      std::memcpy(&init.cmin, &big, sizeof(double));
      *red_host_ = init;
      ACK(cudaMemcpyAsync(red_dev_, red_host_, sizeof(DevReduce), cudaMemcpyHostToDevice, stream_));
      if (flags_)
        k_ingest<T, T, lcsdata_t, true><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, pr_.u[l], pr_.v[l], pr_.w[l], f[0], f[1], f[2],
                                                                                   red_dev_);
      else
        k_ingest<T, T, lcsdata_t, false><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, pr_.u[l], pr_.v[l], pr_.w[l], f[0], f[1], f[2],
                                                                                    red_dev_);
      ACK(cudaGetLastError());
      ACK(cudaMemcpyAsync(red_host_, red_dev_, sizeof(DevReduce), cudaMemcpyDeviceToHost, stream_));
      ACK(cudaStreamSynchronize(stream_));
      if (red_host_->err) {
        msg = "adjoint: non-finite velocity";
        return false;
      }
      std::memcpy(&cmax_[l], &red_host_->cmax, sizeof(double));
    }
    nsub_.assign(L, 0);
    for (int l = 1; l < L; l++) {
      const lcsdata_t dt_f = pr_.times[l] - pr_.times[l - 1];
      const lcsdata_t q = ((lcsdata_t)cmax_[l] * dt_f) / lcsdata_t(pr_.cfl);
      long ns = (long)std::ceil((double)q);
      nsub_[l] = (int)std::max(1L, ns);
    }
    if (!field3(fm_[0], msg) || !field3(fm_[1], msg)) return false;
    if (cubic_) {
      if (!slab(Cl_, (size_t)3 * L, msg)) return false;
      for (int l = 0; l < L; l++) fit3(&U_[3 * l], &Cl_[3 * l]);
      for (int st = 1; st < 4; st++)
        if (!field3(blend_[st], msg)) return false;
      if (!field3(cfm_, msg)) return false;
      ACK(cudaGetLastError());
    }
    if (tangent_) {
      // the direction, padded and ghost-filled like the levels (its CFL maxima are unused)
      if (!slab(DU_, (size_t)3 * L, msg)) return false;
      if (!(red_tan_ = pool_.alloc<DevReduce>(1, msg))) return false;
      ACK(cudaMemsetAsync(red_tan_, 0, sizeof(DevReduce), stream_));
      for (int l = 0; l < L; l++)
        if (flags_)
          k_ingest<T, T, lcsdata_t, true><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, pr_.du[l], pr_.dv[l], pr_.dw[l], DU_[3 * l],
                                                                                     DU_[3 * l + 1], DU_[3 * l + 2], red_tan_);
        else
          k_ingest<T, T, lcsdata_t, false><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, pr_.du[l], pr_.dv[l], pr_.dw[l], DU_[3 * l],
                                                                                      DU_[3 * l + 1], DU_[3 * l + 2], red_tan_);
      ACK(cudaGetLastError());
      int terr = 0;
      ACK(cudaMemcpyAsync(&terr, &red_tan_->err, sizeof(int), cudaMemcpyDeviceToHost, stream_));
      ACK(cudaStreamSynchronize(stream_));
      if (terr) {
        msg = "adjoint: non-finite tangent direction";
        return false;
      }
      if (!field3(dfm_[0], msg) || !field3(dfm_[1], msg)) return false;
      if (cubic_) {
        if (!slab(DC_, (size_t)3 * L, msg)) return false;
        for (int l = 0; l < L; l++) fit3(&DU_[3 * l], &DC_[3 * l]);
        if (!field3(dcfm_, msg)) return false;
        ACK(cudaGetLastError());
      }
    }
    cur_ = 0;
    const int K = pr_.checkpoint_every;
    const int nseg = (L - 2) / K + 1;  // segments of updates 1..L-1
    if (!slab(cp_, (size_t)3 * nseg, msg)) return false;
    for (int l = 1; l < L; l++) {
      if ((l - 1) % K == 0) {
        const int s = (l - 1) / K;
        for (int c = 0; c < 3; c++)
          ACK(cudaMemcpyAsync(cp_[3 * s + c], fm_[cur_][c], ntot_ * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
      }
      if (!advance(l, fm_, cur_, nullptr, msg, tangent_)) return false;
    }
    // FTLE of the final map and J
    T *in[3];
    for (int c = 0; c < 3; c++)
      if (!(in[c] = pool_.alloc<T>(N_, msg))) return false;
    T *ftle = pool_.alloc<T>(N_, msg);
    if (!ftle) return false;
    FieldPtrs<T> src{};
    FieldPtrsW<T> dst{};
    for (int c = 0; c < 3; c++) {
      src.f[c] = fm_[cur_][c];
      dst.f[c] = in[c];
    }
    k_interior<T><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, src, dst);
    FieldPtrs<T> cm{};
    for (int c = 0; c < 3; c++) cm.f[c] = in[c];
    const T Tint = (T)(pr_.times[L - 1] - pr_.times[0]);
    if (flags_) k_ftle<T, T, true><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, cm, ftle, Tint, 0);
    else k_ftle<T, T, false><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, cm, ftle, Tint, 0);
    ACK(cudaGetLastError());
    std::vector<T> hf(N_), hw(N_);
    ACK(cudaMemcpyAsync(hf.data(), ftle, N_ * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    ACK(cudaMemcpyAsync(hw.data(), pr_.weight, N_ * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    ACK(cudaStreamSynchronize(stream_));
    double s = 0.0;
    for (long q = 0; q < N_; q++) s += (double)hw[q] * (double)hf[q];
    *J = s;
    if (tangent_) {
      double *dj = pool_.alloc<double>(N_, msg);
      if (!dj) return false;
      FieldPtrs<T> fm{}, dfm{};
      for (int c = 0; c < 3; c++) {
        fm.f[c] = fm_[cur_][c];
        dfm.f[c] = dfm_[cur_][c];
      }
      k_ftle_tangent<T><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, fm, dfm, pr_.weight, Tint, dj);
      ACK(cudaGetLastError());
      std::vector<double> hd(N_);
      ACK(cudaMemcpyAsync(hd.data(), dj, N_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
      ACK(cudaStreamSynchronize(stream_));
      double t = 0.0;
      for (long q = 0; q < N_; q++) t += hd[q];
      *pr_.dJ = t;
    }
    return true;
  }

  // every subcycle of update l (levels l-1 -> l) on the double buffer buf, starting from
  // buf[cur]; cur follows the result.  With `keep`, the flow map before subcycle q is copied
  // to keep[3 q + c].
  // With `tangent`, the tangent map dfm_ advances alongside (dfm_[cur] pairs with buf[cur]).
  bool advance(int l, T *buf[2][3], int &cur, T *const *keep, std::string &msg, bool tangent = false) {
    const lcsdata_t t0 = pr_.times[l - 1], t1 = pr_.times[l];
    const lcsdata_t dt_f = t1 - t0;
    const int ns = nsub_[l];
    const lcsdata_t dt = lcsdata_t(-1) * (dt_f / (lcsdata_t)ns);
    VelFields<T> V{};
    for (int c = 0; c < 3; c++) {
      V.un[c] = U_[3 * (l - 1) + c];
      V.unp1[c] = U_[3 * l + c];
    }
    lcsdata_t lp = t1;
    for (int q = 0; q < ns; q++) {
      if (keep)
        for (int c = 0; c < 3; c++)
          ACK(cudaMemcpyAsync(keep[3 * q + c], buf[cur][c], ntot_ * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
      const StageTimes S = stage_times(t0, t1, lp, dt);
      FieldPtrs<T> fo{};
      FieldPtrsW<T> fn{};
      for (int c = 0; c < 3; c++) {
        fo.f[c] = buf[cur][c];
        fn.f[c] = buf[cur ^ 1][c];
      }
      const SplineAxes<T> sa{};
      int *err = &red_dev_->err;
      const dim3 grd = node_grid(), blk(32, 8, 1);
      if (cubic_) {
        if (!advance_cubic(l, buf, cur, S, (T)dt, tangent, msg)) return false;
        cur ^= 1;
        lp = lp + dt;
        continue;
      }
      if (tangent) {
        // reads the map before the subcycle, so it runs before the forward kernel replaces it
        VelFields<T> D{};
        FieldPtrs<T> dfo{};
        FieldPtrsW<T> dfn{};
        for (int c = 0; c < 3; c++) {
          D.un[c] = DU_[3 * (l - 1) + c];
          D.unp1[c] = DU_[3 * l + c];
          dfo.f[c] = dfm_[cur][c];
          dfn.f[c] = dfm_[cur ^ 1][c];
        }
        if (flags_) tangent_linear<true>(grd, blk, V, D, fo, dfo, dfn, S, (T)dt, err);
        else tangent_linear<false>(grd, blk, V, D, fo, dfo, dfn, S, (T)dt, err);
        if (!flags_) k_periodic_ghosts<T><<<(unsigned)((ntot_ + 255) / 256), 256, 0, stream_>>>(dg_, dfn, ntot_);
        ACK(cudaGetLastError());
      }
      if (flags_) forward_linear<true>(grd, blk, sa, V, fo, fn, S, (T)dt, err);
      else forward_linear<false>(grd, blk, sa, V, fo, fn, S, (T)dt, err);
      ACK(cudaGetLastError());
      cur ^= 1;
      lp = lp + dt;
    }
    return true;
  }

  // one LINEAR subcycle: the library's kernel, and the tangent sweep's (F: boundary flags)
  template <bool F>
  void forward_linear(dim3 grd, dim3 blk, const SplineAxes<T> &sa, const VelFields<T> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn,
                      const StageTimes &S, T dt, int *err) {
    switch (pr_.integrator) {
      case RK4: k_sl_subcycle<T, T, RK4_, INTERP_LINEAR, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case RK3: k_sl_subcycle<T, T, RK3_, INTERP_LINEAR, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case RK2: k_sl_subcycle<T, T, RK2_, INTERP_LINEAR, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case TRAPEZOIDAL: k_sl_subcycle<T, T, TRAPEZOIDAL_, INTERP_LINEAR, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      default: k_sl_subcycle<T, T, EULER_, INTERP_LINEAR, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
    }
  }
  template <bool F>
  void tangent_linear(dim3 grd, dim3 blk, const VelFields<T> &V, const VelFields<T> &D, FieldPtrs<T> fo, FieldPtrs<T> dfo,
                      FieldPtrsW<T> dfn, const StageTimes &S, T dt, int *err) {
    switch (pr_.integrator) {
      case RK4: k_sl_tangent<T, RK4, F><<<grd, blk, 0, stream_>>>(dg_, V, D, fo, dfo, dfn, S, dt, err); break;
      case RK3: k_sl_tangent<T, RK3, F><<<grd, blk, 0, stream_>>>(dg_, V, D, fo, dfo, dfn, S, dt, err); break;
      case RK2: k_sl_tangent<T, RK2, F><<<grd, blk, 0, stream_>>>(dg_, V, D, fo, dfo, dfn, S, dt, err); break;
      default: k_sl_tangent<T, EULER, F><<<grd, blk, 0, stream_>>>(dg_, V, D, fo, dfo, dfn, S, dt, err); break;
    }
  }
  template <bool F>
  void adjoint_linear(const VelFields<T> &V, FieldPtrs<T> fo, FieldPtrs<T> fbn, FieldPtrsW<T> fbo, FieldPtrsW<T> A1, FieldPtrsW<T> A2,
                      FieldPtrsW<T> A3, const StageTimes &S, T dt) {
    const dim3 grd = node_grid(), blk(32, 8, 1);
    switch (pr_.integrator) {
      case RK4: k_sl_adjoint<T, RK4, F><<<grd, blk, 0, stream_>>>(dg_, V, fo, fbn, fbo, A1, A2, A3, S, dt); break;
      case RK3: k_sl_adjoint<T, RK3, F><<<grd, blk, 0, stream_>>>(dg_, V, fo, fbn, fbo, A1, A2, A3, S, dt); break;
      case RK2: k_sl_adjoint<T, RK2, F><<<grd, blk, 0, stream_>>>(dg_, V, fo, fbn, fbo, A1, A2, A3, S, dt); break;
      default: k_sl_adjoint<T, EULER, F><<<grd, blk, 0, stream_>>>(dg_, V, fo, fbn, fbo, A1, A2, A3, S, dt); break;
    }
  }
  // the adjoint of a ghost fill: periodic images only, or every boundary rule (KIND: the flow map's
  // or the velocity's)
  template <int KIND>
  void fold(FieldPtrsW<T> f) {
    const unsigned nb = (unsigned)((ntot_ + 255) / 256);
    if (!flags_) {
      k_fold_ghosts<T><<<nb, 256, 0, stream_>>>(dg_, f, ntot_);
      return;
    }
    k_fold_copy<T, KIND><<<nb, 256, 0, stream_>>>(dg_, f, ntot_);
    k_fold_zero<T, KIND><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, f);
    k_fold_image<T, KIND><<<nb, 256, 0, stream_>>>(dg_, f, ntot_);
  }

  // one CUBIC subcycle of update l from buf[cur] into buf[cur ^ 1] (and the tangent map along)
  bool advance_cubic(int l, T *buf[2][3], int cur, const StageTimes &S, T dt, bool tangent, std::string &msg) {
    VelFields<T> V{};
    FieldPtrs<T> cn{}, cp{};
    for (int c = 0; c < 3; c++) {
      V.un[c] = U_[3 * (l - 1) + c];
      V.unp1[c] = U_[3 * l + c];
      cn.f[c] = Cl_[3 * (l - 1) + c];
      cp.f[c] = Cl_[3 * l + c];
    }
    // stage blends of the two levels' coefficients, as the library's k_blend forms them
    const int nst = pr_.integrator == RK4 ? 4 : (pr_.integrator == RK3 ? 3 : (pr_.integrator == RK2 ? 2 : 1));
    BlendOut<T> o{};
    int nout = 0;
    for (int st = 1; st < nst; st++) {
      if (pr_.integrator == RK4 && st == 2) {  // the second half-step stage: the first's time, its blend
        for (int c = 0; c < 3; c++) V.cs[2][c] = blend_[1][c];
        continue;
      }
      const T ct = (T)S.ct[st];
      for (int c = 0; c < 3; c++) {
        o.f[nout][c] = blend_[st][c];
        V.cs[st][c] = blend_[st][c];
      }
      o.omc[nout] = T(1) - ct;
      o.ct[nout] = ct;
      nout++;
    }
    if (nout > 0) {
      const long npair = (ntot_ + 1) / 2;
      k_blend<T><<<dim3((unsigned)((npair + 255) / 256), 3), 256, 0, stream_>>>(cn, cp, o, nout, ntot_);
    }
    fit3(buf[cur], cfm_);
    FieldPtrs<T> fo{};
    FieldPtrsW<T> fn{};
    for (int c = 0; c < 3; c++) {
      fo.f[c] = cfm_[c];
      fn.f[c] = buf[cur ^ 1][c];
    }
    if (tangent) {
      fit3(dfm_[cur], dcfm_);
      VelFields<T> D{};
      FieldPtrs<T> dcn{}, dcp{}, dcf{};
      FieldPtrsW<T> dfn{};
      for (int c = 0; c < 3; c++) {
        D.un[c] = DU_[3 * (l - 1) + c];
        D.unp1[c] = DU_[3 * l + c];
        dcn.f[c] = DC_[3 * (l - 1) + c];
        dcp.f[c] = DC_[3 * l + c];
        dcf.f[c] = dcfm_[c];
        dfn.f[c] = dfm_[cur ^ 1][c];
      }
      const dim3 g4 = node_grid4(), b4(32, 4, 1);
      if (pr_.integrator == RK4) k_sl_tangent_cubic<T, RK4><<<g4, b4, 0, stream_>>>(dg_, sa_, V, D, cn, cp, dcn, dcp, fo, dcf, dfn, S, dt);
      else if (pr_.integrator == RK3) k_sl_tangent_cubic<T, RK3><<<g4, b4, 0, stream_>>>(dg_, sa_, V, D, cn, cp, dcn, dcp, fo, dcf, dfn, S, dt);
      else if (pr_.integrator == RK2) k_sl_tangent_cubic<T, RK2><<<g4, b4, 0, stream_>>>(dg_, sa_, V, D, cn, cp, dcn, dcp, fo, dcf, dfn, S, dt);
      else k_sl_tangent_cubic<T, EULER><<<g4, b4, 0, stream_>>>(dg_, sa_, V, D, cn, cp, dcn, dcp, fo, dcf, dfn, S, dt);
      k_periodic_ghosts<T><<<(unsigned)((ntot_ + 255) / 256), 256, 0, stream_>>>(dg_, dfn, ntot_);
    }
    int *err = &red_dev_->err;
    const dim3 grd = node_grid(), blk(32, 8, 1);
    if (pr_.integrator == RK4)
      k_sl_subcycle<T, T, RK4_, INTERP_SPLINE4, false><<<grd, blk, 0, stream_>>>(dg_, sa_, V, fo, fn, S, dt, err);
    else if (pr_.integrator == RK3)
      k_sl_subcycle<T, T, RK3_, INTERP_SPLINE4, false><<<grd, blk, 0, stream_>>>(dg_, sa_, V, fo, fn, S, dt, err);
    else if (pr_.integrator == RK2)
      k_sl_subcycle<T, T, RK2_, INTERP_SPLINE4, false><<<grd, blk, 0, stream_>>>(dg_, sa_, V, fo, fn, S, dt, err);
    else if (pr_.integrator == TRAPEZOIDAL)
      k_sl_subcycle<T, T, TRAPEZOIDAL_, INTERP_SPLINE4, false><<<grd, blk, 0, stream_>>>(dg_, sa_, V, fo, fn, S, dt, err);
    else
      k_sl_subcycle<T, T, EULER_, INTERP_SPLINE4, false><<<grd, blk, 0, stream_>>>(dg_, sa_, V, fo, fn, S, dt, err);
    ACK(cudaGetLastError());
    return true;
  }

  bool backward(std::string &msg) {
    const int L = pr_.nlevels, K = pr_.checkpoint_every;
    if (!slab(Ub_, (size_t)3 * L, msg)) return false;
    if (cubic_ && !slab(Cb_, (size_t)3 * L, msg)) return false;
    T *fbar[2][3];
    if (!field3(fbar[0], msg) || !field3(fbar[1], msg)) return false;
    int fb = 0;
    // FTLE adjoint of the final map
    {
      FieldPtrs<T> fm{};
      FieldPtrsW<T> out{};
      for (int c = 0; c < 3; c++) {
        fm.f[c] = fm_[cur_][c];
        out.f[c] = fbar[fb][c];
      }
      const T Tint = (T)(pr_.times[L - 1] - pr_.times[0]);
      k_ftle_adjoint<T><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, fm, pr_.weight, Tint, out);
      ACK(cudaGetLastError());
    }
    const long nb = (ntot_ + 255) / 256;
    const int nseg = (L - 2) / K + 1;
    // per-subcycle velocity adjoints of the stages (zero between subcycles; a third for RK3)
    FieldPtrsW<T> A1{}, A2{}, A3{};
    {
      T *a[3], *b[3], *e[3];
      if (!field3(a, msg) || !field3(b, msg)) return false;
      const bool three = pr_.integrator == RK3 || pr_.integrator == RK4;
      if (three && !field3(e, msg)) return false;
      for (int c = 0; c < 3; c++) {
        A1.f[c] = a[c];
        A2.f[c] = b[c];
        A3.f[c] = three ? e[c] : nullptr;
      }
    }
    // flow maps before every subcycle of the largest segment
    int maxsub = 0;
    for (int s = 0; s < nseg; s++) {
      int m = 0;
      for (int l = s * K + 1; l <= std::min((s + 1) * K, L - 1); l++) m += nsub_[l];
      maxsub = std::max(maxsub, m);
    }
    std::vector<T *> states;
    if (!slab(states, (size_t)3 * maxsub, msg)) return false;
    T *work[2][3];
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 3; c++) work[b][c] = fm_[b][c];  // the forward buffers are free now
    for (int s = nseg - 1; s >= 0; s--) {
      const int l0 = s * K + 1, l1 = std::min((s + 1) * K, L - 1);
      // recompute the segment from its checkpoint, keeping the flow map before each subcycle
      std::vector<int> first(l1 - l0 + 2, 0);
      for (int l = l0; l <= l1; l++) first[l - l0 + 1] = first[l - l0] + nsub_[l];
      for (int c = 0; c < 3; c++) ACK(cudaMemcpyAsync(work[0][c], cp_[3 * s + c], ntot_ * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
      int wc = 0;
      for (int l = l0; l <= l1; l++)
        if (!advance(l, work, wc, &states[(size_t)3 * first[l - l0]], msg)) return false;
      // reverse through the segment
      for (int l = l1; l >= l0; l--) {
        const lcsdata_t t0 = pr_.times[l - 1], t1 = pr_.times[l];
        const int ns = nsub_[l];
        const lcsdata_t dt = lcsdata_t(-1) * ((t1 - t0) / (lcsdata_t)ns);
        std::vector<lcsdata_t> lps(ns);
        lcsdata_t lp = t1;
        for (int q = 0; q < ns; q++) {
          lps[q] = lp;
          lp = lp + dt;
        }
        VelFields<T> V{};
        FieldPtrsW<T> ubn{}, ubp{};
        for (int c = 0; c < 3; c++) {
          V.un[c] = U_[3 * (l - 1) + c];
          V.unp1[c] = U_[3 * l + c];
          ubn.f[c] = Ub_[3 * (l - 1) + c];
          ubp.f[c] = Ub_[3 * l + c];
        }
        for (int q = ns - 1; q >= 0; q--) {
          // the new map's ghosts were copies of its interior
          FieldPtrsW<T> fw{};
          for (int c = 0; c < 3; c++) fw.f[c] = fbar[fb][c];
          fold<GHOST_FM>(fw);
          for (int c = 0; c < 3; c++) ACK(cudaMemsetAsync(fbar[fb ^ 1][c], 0, ntot_ * sizeof(T), stream_));
          FieldPtrs<T> fo{}, fbn{};
          FieldPtrsW<T> fbo{};
          for (int c = 0; c < 3; c++) {
            fo.f[c] = states[(size_t)3 * (first[l - l0] + q) + c];
            fbn.f[c] = fbar[fb][c];
            fbo.f[c] = fbar[fb ^ 1][c];
          }
          const StageTimes S = stage_times(t0, t1, lps[q], dt);
          // the stage whose adjoint field a3 holds: the third (RK3) or the fourth (RK4); RK4's two
          // half-step stages share ct[1] = ct[2] and a2
          const int last = pr_.integrator == RK4 ? 3 : 2;
          if (cubic_) {
            fit3(&states[(size_t)3 * (first[l - l0] + q)], cfm_);
            FieldPtrs<T> cn{}, cp{}, cf{};
            FieldPtrsW<T> cbn{}, cbp{};
            for (int c = 0; c < 3; c++) {
              cn.f[c] = Cl_[3 * (l - 1) + c];
              cp.f[c] = Cl_[3 * l + c];
              cf.f[c] = cfm_[c];
              cbn.f[c] = Cb_[3 * (l - 1) + c];
              cbp.f[c] = Cb_[3 * l + c];
            }
            const dim3 g4 = node_grid4(), b4(32, 4, 1);
            if (pr_.integrator == RK4)
              k_sl_adjoint_cubic<T, RK4><<<g4, b4, 0, stream_>>>(dg_, sa_, V, cn, cp, cf, fbn, fbo, A1, A2, A3, S, (T)dt);
            else if (pr_.integrator == RK3)
              k_sl_adjoint_cubic<T, RK3><<<g4, b4, 0, stream_>>>(dg_, sa_, V, cn, cp, cf, fbn, fbo, A1, A2, A3, S, (T)dt);
            else if (pr_.integrator == RK2)
              k_sl_adjoint_cubic<T, RK2><<<g4, b4, 0, stream_>>>(dg_, sa_, V, cn, cp, cf, fbn, fbo, A1, A2, A3, S, (T)dt);
            else
              k_sl_adjoint_cubic<T, EULER><<<g4, b4, 0, stream_>>>(dg_, sa_, V, cn, cp, cf, fbn, fbo, A1, A2, A3, S, (T)dt);
            // the previous map's adjoint was scattered in coefficient space: through the fit
            fitT3(fbar[fb ^ 1]);
            if (pr_.integrator == RK3 || pr_.integrator == RK4)
              k_distribute_cubic<T, true><<<dim3((unsigned)nb, 3), 256, 0, stream_>>>(A1, A2, A3, ubn, ubp, cbn, cbp, (T)S.ct[0], (T)S.ct[1],
                                                                                        (T)S.ct[last], ntot_);
            else
              k_distribute_cubic<T, false><<<dim3((unsigned)nb, 3), 256, 0, stream_>>>(A1, A2, A3, ubn, ubp, cbn, cbp, (T)S.ct[0],
                                                                                         (T)S.ct[1], T(0), ntot_);
            ACK(cudaGetLastError());
            fb ^= 1;
            continue;
          }
          if (flags_) adjoint_linear<true>(V, fo, fbn, fbo, A1, A2, A3, S, (T)dt);
          else adjoint_linear<false>(V, fo, fbn, fbo, A1, A2, A3, S, (T)dt);
          if (pr_.integrator == RK3 || pr_.integrator == RK4)
            k_distribute<T, true><<<dim3((unsigned)nb, 3), 256, 0, stream_>>>(A1, A2, A3, ubn, ubp, (T)S.ct[0], (T)S.ct[1], (T)S.ct[last],
                                                                             ntot_);
          else
            k_distribute<T, false><<<dim3((unsigned)nb, 3), 256, 0, stream_>>>(A1, A2, A3, ubn, ubp, (T)S.ct[0], (T)S.ct[1], T(0),
                                                                              ntot_);
          ACK(cudaGetLastError());
          fb ^= 1;
        }
      }
    }
    // velocity ghosts were copies of the ingested interior: fold, then hand out (CUBIC: the
    // coefficient-space adjoint of each level through its fit first)
    for (int l = 0; l < L; l++) {
      FieldPtrsW<T> f{};
      FieldPtrs<T> fr{};
      for (int c = 0; c < 3; c++) {
        f.f[c] = Ub_[3 * l + c];
        fr.f[c] = Ub_[3 * l + c];
      }
      if (cubic_) {
        fitT3(&Cb_[3 * l]);
        FieldPtrs<T> cb{};
        for (int c = 0; c < 3; c++) cb.f[c] = Cb_[3 * l + c];
        k_add3<T><<<dim3((unsigned)nb, 3), 256, 0, stream_>>>(f, cb, ntot_);
      }
      fold<GHOST_VEL>(f);
      k_grad_out<T><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, fr, pr_.gu[l], pr_.gv[l], pr_.gw[l]);
      ACK(cudaGetLastError());
    }
    return true;
  }


  // CUBIC: spline axes, transposed pull tables, coefficient levels (and their adjoints and
  // tangents), the stage blends and the previous map's coefficients of one subcycle
  bool cubic_ = false;
  bool flags_ = false;  // boundary flags (walls, slip, inflow / outflow, masks, 2-D)
  SplineAxes<T> sa_{};
  T *ptr_[3] = {nullptr, nullptr, nullptr};
  std::vector<T *> Cl_, Cb_, DC_;
  T *blend_[4][3] = {};
  T *cfm_[3] = {nullptr, nullptr, nullptr};
  T *dcfm_[3] = {nullptr, nullptr, nullptr};

  // coefficients of the padded fields src into dst (the library's fit: x, then y, then z)
  void fit3(T *const src[3], T *const dst[3]) {
    FieldPtrs<T> s{}, di{};
    FieldPtrsW<T> d{};
    for (int c = 0; c < 3; c++) {
      s.f[c] = src[c];
      di.f[c] = dst[c];
      d.f[c] = dst[c];
    }
    const int sx = dg_.P.sx, sxy = dg_.P.sxy, ny = dg_.P.n[1] + 2, nz = dg_.P.n[2] + 2;
    const long warps = (long)((ny + 31) / 32) * nz;
    const size_t smem = sizeof(T) * 4 * 2 * 32 * (XFIT_W + 1);
    k_fit_xlines<T, 4><<<dim3((unsigned)((warps + 3) / 4), 3), 128, smem, stream_>>>(sa_.ax[0], s, d, ny, nz, (long)sx, (long)sxy);
    k_fit_lines<T, 4><<<dim3((unsigned)(((long)sx * nz + 255) / 256), 3), 256, 0, stream_>>>(sa_.ax[1], di, d, sx, (long)sx * nz,
                                                                                             (long)sx, (long)sxy);
    k_fit_lines<T, 4><<<dim3((unsigned)(((long)sxy + 255) / 256), 3), 256, 0, stream_>>>(sa_.ax[2], di, d, sxy, (long)sxy, (long)sxy,
                                                                                         (long)sxy);
  }

  // adjoint of fit3, in place: the transposed passes z, then y, then x
  void fitT3(T *const f[3]) {
    FieldPtrsW<T> d{};
    for (int c = 0; c < 3; c++) d.f[c] = f[c];
    const long sx = dg_.P.sx, sxy = dg_.P.sxy;
    const int ny = dg_.P.n[1] + 2, nz = dg_.P.n[2] + 2;
    k_fit_transpose<T><<<dim3((unsigned)((sxy + 255) / 256), 3), 256, 0, stream_>>>(ptr_[2], sa_.ax[2].n, d, (int)sxy, sxy, 1L, sxy, sxy);
    k_fit_transpose<T><<<dim3((unsigned)((sx * nz + 255) / 256), 3), 256, 0, stream_>>>(ptr_[1], sa_.ax[1].n, d, (int)sx, sx * nz, 1L, sxy,
                                                                                        sx);
    k_fit_transpose<T><<<dim3((unsigned)(((long)ny * nz + 255) / 256), 3), 256, 0, stream_>>>(ptr_[0], sa_.ax[0].n, d, ny, (long)ny * nz,
                                                                                              sx, sxy, 1L);
  }

  dim3 node_grid4() const { return dim3((dg_.P.n[0] + 31) / 32, (dg_.P.n[1] + 3) / 4, dg_.P.n[2]); }

  const AdjointProblem &pr_;
  HostGrid<lcsdata_t> hg_;
  DevGrid<T> dg_{};
  Pool pool_;
  cudaStream_t stream_ = nullptr;
  DevReduce *red_host_ = nullptr, *red_dev_ = nullptr;
  long N_ = 0, ntot_ = 0;
  std::vector<T *> U_, Ub_, cp_;
  std::vector<double> cmax_;
  std::vector<int> nsub_;
  T *fm_[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int cur_ = 0;
  // tangent-linear sweep: direction levels (padded) and the tangent map's double buffer
  bool tangent_ = false;
  std::vector<T *> DU_;
  T *dfm_[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  DevReduce *red_tan_ = nullptr;
};

}  // namespace

bool adjoint_ftle(const AdjointProblem &p, double *J, std::string &msg) {
  Adjoint<lcsdata_t> a(p);
  return a.run(J, msg);
}

}  // namespace cfd2lcs
