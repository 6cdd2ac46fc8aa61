// __global__ kernels of libcfd2lcs_b200.  One thread per grid node or per particle; the
// fields are ghost-padded SoA arrays (src/structured_m.f90:73-96 layout, i fastest).
#pragma once

#include <cfloat>

#include "advect.cuh"

namespace cfd2lcs {

// Interior node of this thread; false for threads past the grid.
__device__ __forceinline__ bool node_of_thread(const int n[3], int &i, int &j, int &k) {
  i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  k = blockIdx.z * blockDim.z + threadIdx.z + 1;
  return i <= n[0] && j <= n[1] && k <= n[2];
}

__device__ __forceinline__ int interior_index(const int n[3], int i, int j, int k) {
  return (i - 1) + n[0] * ((j - 1) + n[1] * (k - 1));
}

// CFL reduction result and the device error word (one small struct read back per update).
struct DevReduce {
  unsigned long long cmax;  // bits of the largest sum_i |u_i| / delta_i (non-negative double)
  unsigned long long cmin;  // bits of the smallest
  int err;
  int pad;
};

template <typename T>
__device__ __forceinline__ T inv_half_span(const DevGrid<T> &g, int a, int i, int j, int k) {
  // class bits of the other two axes (b = a+1, c = a+2 mod 3), see HostGrid::invd
  const int idx[3] = {i, j, k};
  const int b = (a + 1) % 3, c = (a + 2) % 3;
  const int cb = (idx[b] - 1 == 0 ? 1 : 0) | (idx[b] + 1 == g.P.n[b] + 1 ? 2 : 0);
  const int cc = (idx[c] - 1 == 0 ? 1 : 0) | (idx[c] + 1 == g.P.n[c] + 1 ? 2 : 0);
  return __ldg(g.invd[a] + ((size_t)idx[a] * 4 + cb) * 4 + cc);
}

// ---------------------------------------------------------------------------------------
// K0  velocity ingest: u_np1 = caller's (u,v,w) on the padded layout, exchange_sdata SELF
// copies + set_velocity_bc as ghost writes (src/cfd2lcs.f90:112-117), and the CFL maximum
// of set_dt (src/lp_motion_m.f90:86-98) as a block reduction plus atomics.
// ---------------------------------------------------------------------------------------
// T: grid / interface type (lcsdata_t); TV: velocity storage type.  The CFL number is
// computed from the caller's values in the interface precision, so the subcycle count does
// not depend on the storage type.
template <typename T, typename TV, typename U, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_ingest(DevGrid<T> g, const U *__restrict__ su, const U *__restrict__ sv,
                                                 const U *__restrict__ sw, TV *u0, TV *u1, TV *u2, DevReduce *red) {
  int i, j, k;
  const bool ok = node_of_thread(g.P.n, i, j, k);
  double c = 0.0;
  bool bad = false;
  if (ok) {
    const int s = interior_index(g.P.n, i, j, k);
    const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
    T in[3] = {T(su[s]), T(sv[s]), T(sw[s])};
    const bool masked = HAS_FLAGS && g.flag[p] == LCS_MASK;
    if (masked) in[0] = in[1] = in[2] = T(0);
    TV vpre[3] = {TV(su[s]), TV(sv[s]), TV(sw[s])};
    TV vfin[3] = {TV(in[0]), TV(in[1]), TV(in[2])};
    u0[p] = vfin[0];
    u1[p] = vfin[1];
    u2[p] = vfin[2];
    TV *const f[3] = {u0, u1, u2};
    write_ghosts<T, HAS_FLAGS, GHOST_VEL, TV>(g, f, i, j, k, vpre, vfin, &red->err);
    T cf = T(0);
    cf = cf + fabs(in[0] * inv_half_span(g, 0, i, j, k));
    cf = cf + fabs(in[1] * inv_half_span(g, 1, i, j, k));
    cf = cf + fabs(in[2] * inv_half_span(g, 2, i, j, k));
    c = (double)cf;
    bad = !(c <= DBL_MAX);
  }
  double cmax = ok && !bad ? c : 0.0, cmin = ok && !bad ? c : DBL_MAX;
  if (bad) atomicOr(&red->err, ERR_NONFINITE_VELOCITY);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    cmin = fmin(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
  }
  __shared__ double smax[8], smin[8];
  const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
  const int wid = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
  if (lane == 0) {
    smax[wid] = cmax;
    smin[wid] = cmin;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    cmax = lane < nw ? smax[lane] : 0.0;
    cmin = lane < nw ? smin[lane] : DBL_MAX;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
      cmin = fmin(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
    }
    if (lane == 0) {
      atomicMax(&red->cmax, (unsigned long long)__double_as_longlong(cmax));
      atomicMin(&red->cmin, (unsigned long long)__double_as_longlong(cmin));
    }
  }
}

// ---------------------------------------------------------------------------------------
// K1  one backward semi-Lagrangian subcycle, fused (src/flowmap_m.f90:71-97):
// integrate the grid point back by dt with the stage velocities of integrate_lp, project
// and apply the particle BC, sample the previous flow map at the departure point, write
// fm_new = (fm_old(x_dep) + (x_dep - x_grid)) * mask, then the flow-map ghost ring
// (exchange_sdata + set_flowmap_bc) from the boundary threads.
// ---------------------------------------------------------------------------------------
template <typename T, typename TV, int INTEG, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_sl_subcycle(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, FieldPtrs<T> fmo,
                                                      FieldPtrsW<T> fmn, StageTimes S, T dt, int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const T x0[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  int no[3] = {i, j, k};
  T x[3];
  integrate<T, TV, INTEG, INTERP>(g, sa, V, S, dt, x0, no, x);
  project_plane(g, no, x);
  const bool stick = particle_bc<T, HAS_FLAGS>(g, no, x, err);
  if (stick) {
    x[0] = x0[0];
    x[1] = x0[1];
    x[2] = x0[2];
  }
  T fmp[3];
  const int nod[3] = {i, j, k};
  sample_field<T, INTERP>(g, sa, fmo.f, x, nod, fmp);
  const int fl = HAS_FLAGS ? (int)g.flag[p] : (int)LCS_INTERNAL;
  const T mask = fl != LCS_MASK ? T(1) : T(0);
  T vpre[3], vfin[3];
  const bool zero = HAS_FLAGS && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    vpre[c] = (fmp[c] + (x[c] - x0[c])) * mask;
    vfin[c] = zero ? T(0) : vpre[c];
    fmn.f[c][p] = vfin[c];
  }
  write_ghosts<T, HAS_FLAGS, GHOST_FM>(g, fmn.f, i, j, k, vpre, vfin, err);
}

// ---------------------------------------------------------------------------------------
// K6  one forward particle subcycle (update_lp, src/lp_motion_m.f90:15-54): integrate,
// project, BC, stick, accumulate the displacement, one pass of the node search and the
// periodic wrap of exchange_lpdata.  Particle q starts at interior node q.
// ---------------------------------------------------------------------------------------
template <typename T, typename TV, int INTEG, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_fwd_subcycle(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, Particles<T> P, StageTimes S,
                                                       T dt, int np, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  T xn[3] = {P.x[0][q], P.x[1][q], P.x[2][q]};
  int no[3] = {P.no[0][q], P.no[1][q], P.no[2][q]};
  T x[3];
  integrate<T, TV, INTEG, INTERP>(g, sa, V, S, dt, xn, no, x);
  project_plane(g, no, x);
  const bool stick = particle_bc<T, HAS_FLAGS>(g, no, x, err);
  if (stick) {
    x[0] = xn[0];
    x[1] = xn[1];
    x[2] = xn[2];
  }
#pragma unroll
  for (int c = 0; c < 3; c++) P.dx[c][q] = P.dx[c][q] + (x[c] - xn[c]);
  track_pass(g, x, no);
  wrap_particle(g, x, no);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    P.x[c][q] = x[c];
    P.no[c][q] = no[c];
  }
}

// ---------------------------------------------------------------------------------------
// K7  ring snapshot (write_flowmap_substep, src/flowmap_m.f90:106-156, and the exchange +
// set_flowmap_bc the reconstruction applies after reading a slot back, :276-278): interior
// values from the working flow map (backward) or from the particle displacements (forward,
// exchange_lpmap fm(no0) = dx), ghosts by the flow-map rule.
// ---------------------------------------------------------------------------------------
template <typename T, bool HAS_FLAGS, bool FROM_DX>
__global__ void __launch_bounds__(256) k_snapshot(DevGrid<T> g, FieldPtrs<T> src, Particles<T> P, FieldPtrsW<T> dst, int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  T v[3];
  if (FROM_DX) {
    const int q = interior_index(g.P.n, i, j, k);
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = P.dx[c][q];
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = src.f[c][p];
  }
  const int fl = HAS_FLAGS ? (int)g.flag[p] : (int)LCS_INTERNAL;
  const bool zero = HAS_FLAGS && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
  T vfin[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    vfin[c] = zero ? T(0) : v[c];
    dst.f[c][p] = vfin[c];
  }
  // the slot is re-padded from its interior, which already carries the zeroing
  write_ghosts<T, HAS_FLAGS, GHOST_FM>(g, dst.f, i, j, k, vfin, vfin, err);
}

// ---------------------------------------------------------------------------------------
// K4  composition of the sub-flow maps (reconstruct_flowmap, src/flowmap_m.f90:158-323):
// per lcs node, walk the listed slots, x += fm_s(x), accumulate the displacement, wrap with
// exchange_lp_alltoall's bounding-box/periodic-image rule (src/comms_m.f90:1421-1476,
// :1609-1655) and re-locate the node with the recursive search (tracking with the forward
// wrap).  Output: the composed map (exchange_lpmap) after the interior flow-map BC.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void alltoall_wrap(const DevGrid<T> &g, T x[3], int no[3]) {
  const T *bb = g.P.bb;
  bool inside = x[0] >= bb[0] && x[0] <= bb[3] && x[1] >= bb[1] && x[1] <= bb[4] && x[2] >= bb[2] && x[2] <= bb[5];
  if (!inside) {
    for (int d = 0; d < 27 && !inside; d++) {  // k outer, j, i inner: index (dk+1)*9+(dj+1)*3+(di+1)
      const T *s = g.P.ps[d];
      const T a = x[0] - s[0], b = x[1] - s[1], c = x[2] - s[2];
      if (a >= bb[0] && a <= bb[3] && b >= bb[1] && b <= bb[4] && c >= bb[2] && c <= bb[5]) {
        x[0] = a;
        x[1] = b;
        x[2] = c;
        inside = true;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const T s = clamp01((x[a] - bb[a]) / (bb[a + 3] - bb[a]));
    const int v = (int)round(T(g.P.n[a]) * s);  // nint(real(n)*s): half away from zero
    no[a] = min(max(v, 1), g.P.n[a]);
  }
}

template <typename T, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_compose(DevGrid<T> g, SplineAxes<T> sa, const T *const *slots, int nsl, FieldPtrsW<T> out,
                                                  int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  T x[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
  int no[3] = {i, j, k};
  T d[3] = {T(0), T(0), T(0)};
  for (int m = 0; m < nsl; m++) {
    const T *const f[3] = {slots[3 * m], slots[3 * m + 1], slots[3 * m + 2]};
    project_plane(g, no, x);
    particle_bc<T, HAS_FLAGS>(g, no, x, err);
    T up[3];
    sample_field<T, INTERP>(g, sa, f, x, no, up);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x[c] + up[c];
      d[c] = d[c] + up[c];
    }
    alltoall_wrap(g, x, no);
    int passes = 0;
    while (true) {
      const bool moved = track_pass(g, x, no);
      passes++;
      if (passes > g.P.maxtrack) {
        atomicOr(err, ERR_TRACKING);
        break;
      }
      wrap_particle(g, x, no);
      if (!moved) break;
    }
  }
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  const int fl = HAS_FLAGS ? (int)g.flag[p] : (int)LCS_INTERNAL;
  const bool zero = HAS_FLAGS && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
  const int q = interior_index(g.P.n, i, j, k);
#pragma unroll
  for (int c = 0; c < 3; c++) out.f[c][q] = zero ? T(0) : d[c];
}

// ---------------------------------------------------------------------------------------
// K5  FTLE (compute_ftle, src/lcs_m.f90:66-193 with grad_sr1, src/gradient_m.f90:11-66):
// central differences of the composed displacement map (face ghosts: periodic image, or
// the flow-map ghost rule), right Cauchy-Green tensor of the displacement gradient in
// FP64, largest eigenvalue by cyclic Jacobi, ftle = log(max(sqrt(lam), tiny))/T.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double eig3_max(double a00, double a01, double a02, double a11, double a12, double a22) {
  double a[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
  for (int sweep = 0; sweep < 32; sweep++) {
    const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
    if (off == 0.0 || off <= 1e-18 * diag) break;
#pragma unroll
    for (int pq = 0; pq < 3; pq++) {
      const int pp = pq == 2 ? 1 : 0, qq = pq == 0 ? 1 : 2;
      const double apq = a[pp][qq];
      if (apq == 0.0) continue;
      const double theta = (a[qq][qq] - a[pp][pp]) / (2.0 * apq);
      const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = rsqrt(t * t + 1.0), s = t * c;
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const double arp = a[r][pp], arq = a[r][qq];
        a[r][pp] = c * arp - s * arq;
        a[r][qq] = s * arp + c * arq;
      }
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const double apr = a[pp][r], aqr = a[qq][r];
        a[pp][r] = c * apr - s * aqr;
        a[qq][r] = s * apr + c * aqr;
      }
    }
  }
  return fmax(fmax(a[0][0], a[1][1]), a[2][2]);
}

template <typename T, typename R, bool HAS_FLAGS>
__device__ __forceinline__ T fm_neighbour(const DevGrid<T> &g, const T *__restrict__ f, int a, int i, int j, int k, int step) {
  int idx[3] = {i, j, k};
  idx[a] += step;
  const int n = g.P.n[a];
  if (idx[a] >= 1 && idx[a] <= n) return __ldg(f + interior_index(g.P.n, idx[0], idx[1], idx[2]));
  if (g.P.per[a]) {  // compute_ftle's face exchange re-copies the periodic image
    idx[a] = idx[a] < 1 ? idx[a] + n : idx[a] - n;
    return __ldg(f + interior_index(g.P.n, idx[0], idx[1], idx[2]));
  }
  if (!HAS_FLAGS) return T(0);
  const int rule = ghost_rule(GHOST_FM, (int)g.flag[pidx(g.P.sx, g.P.sxy, idx[0], idx[1], idx[2])]);
  if (rule == 2) return __ldg(f + interior_index(g.P.n, i, j, k));
  return T(0);
}

template <typename T, typename R, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_ftle(DevGrid<T> g, FieldPtrs<T> fm, R *__restrict__ ftle, R Tint, int incompressible) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  double G[3][3];  // G[c][a] = d fm_c / d x_a
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (g.P.n[a] == 1) {
#pragma unroll
      for (int c = 0; c < 3; c++) G[c][a] = 0.0;
      continue;
    }
    const int idx[3] = {i, j, k};
    const double den = (double)(__ldg(g.lt[a] + idx[a] + 1) - __ldg(g.lt[a] + idx[a] - 1));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T fp = fm_neighbour<T, R, HAS_FLAGS>(g, fm.f[c], a, i, j, k, +1);
      const T fq = fm_neighbour<T, R, HAS_FLAGS>(g, fm.f[c], a, i, j, k, -1);
      G[c][a] = (double)(fp - fq) / den;
    }
  }
  double C[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) C[a][b] = G[0][a] * G[0][b] + G[1][a] * G[1][b] + G[2][a] * G[2][b];
  const double lam = eig3_max(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
  const R sq = sqrt((R)lam);
  const R tiny = sizeof(R) == 8 ? (R)DBL_MIN : (R)FLT_MIN;
  const R mx = sq > tiny ? sq : tiny;  // max(sqrt(W3), tiny): NaN yields tiny
  R v = log(mx) / Tint;
  if (incompressible) v = v > R(0) ? v : R(0);
  ftle[interior_index(g.P.n, i, j, k)] = v;
}

// Reset of forward particles to their grid nodes (reset_lp, src/lp_m.f90:228-294).
template <typename T>
__global__ void k_reset_particles(DevGrid<T> g, Particles<T> P) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int q = interior_index(g.P.n, i, j, k);
  const int nd[3] = {i, j, k};
  const T x[3] = {__ldg(g.lt[0] + i), __ldg(g.lt[1] + j), __ldg(g.lt[2] + k)};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    P.x[c][q] = x[c];
    P.dx[c][q] = T(0);
    P.no[c][q] = nd[c];
  }
}

// Time blend of two padded coefficient fields for one RK stage: c = (1-ct) a + ct b.
template <typename T>
__global__ void __launch_bounds__(256) k_blend(FieldPtrs<T> a, FieldPtrs<T> b, FieldPtrsW<T> c, T omc, T ct, long ntot) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntot) return;
  const int comp = blockIdx.y;
  c.f[comp][q] = omc * __ldg(a.f[comp] + q) + ct * __ldg(b.f[comp] + q);
}

// ---------------------------------------------------------------------------------------
// B-spline fit: banded solves along one axis for every line of the padded field (the three
// dbtpcf passes of db3ink, src/bspline/bspline_sub_module.f90:451-533), one lane per line,
// pull-form forward and backward sweeps (pull_forward / pull_backward).  The first pass of
// a fit reads the source field and writes the coefficient field (the copy db3ink makes is
// fused in); the later passes run in place (src == dst).
// ---------------------------------------------------------------------------------------
// y and z passes: lines start at adjacent addresses (consecutive i), so element e of 32 lines
// is one coalesced row.  Line L starts at L % nfast + (L / nfast) * so; elements es apart.
// Loads are issued G at a time ahead of the dependent sweep.
template <typename T, int K>
__global__ void __launch_bounds__(256) k_fit_lines(SplineAxis<T> A, FieldPtrs<T> src, FieldPtrsW<T> dst, int nfast, long nlines,
                                                    long es, long so) {
  const long L = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlines) return;
  const long off = L % nfast + (L / nfast) * so;
  const T *s = src.f[blockIdx.y] + off;
  T *d = dst.f[blockIdx.y] + off;
  const int n = A.n;
  const T *pc = A.pull;
  constexpr int G = 8;
  T win[3] = {T(0), T(0), T(0)};
  for (int i0 = 0; i0 < n; i0 += G) {
    T v[G];
#pragma unroll
    for (int g = 0; g < G; g++) v[g] = (i0 + g < n) ? s[(long)(i0 + g) * es] : T(0);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i0 + g < n) v[g] = pull_forward<T, K>(pc, i0 + g, v[g], win);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i0 + g < n) d[(long)(i0 + g) * es] = v[g];
  }
  win[0] = win[1] = win[2] = T(0);
  for (int i1 = n - 1; i1 >= 0; i1 -= G) {
    T v[G];
#pragma unroll
    for (int g = 0; g < G; g++) v[g] = (i1 - g >= 0) ? d[(long)(i1 - g) * es] : T(0);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i1 - g >= 0) v[g] = pull_backward<T, K>(pc, i1 - g, v[g], win);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i1 - g >= 0) d[(long)(i1 - g) * es] = v[g];
  }
}

// x pass: lines are contiguous.  One warp per 32 lines (consecutive j at one k): each chunk of
// 32 elements of the 32 lines is staged through a shared tile with coalesced row loads,
// swept by one lane per line inside the tile, and written back with coalesced row stores.
template <typename T, int K>
__global__ void __launch_bounds__(128) k_fit_xlines(SplineAxis<T> A, FieldPtrs<T> src, FieldPtrsW<T> dst, int ny, int nz, long sx,
                                                     long sxy) {
  __shared__ T tile[4][32][33];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int nbf = (ny + 31) / 32;
  const long gw = (long)blockIdx.x * 4 + wp;
  if (gw >= (long)nbf * nz) return;  // warp-uniform
  const int j0 = (int)(gw % nbf) * 32;
  const int nl = min(32, ny - j0);
  const long base = (long)j0 * sx + (gw / nbf) * sxy;
  const T *s = src.f[blockIdx.y] + base;
  T *d = dst.f[blockIdx.y] + base;
  T(*t)[33] = tile[wp];
  const int n = A.n;
  const T *pc = A.pull;
  T win[3] = {T(0), T(0), T(0)};
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int ne = min(32, n - c0);
    if (lane < ne) {
#pragma unroll 8
      for (int r = 0; r < nl; r++) t[r][lane] = s[(long)r * sx + c0 + lane];
    }
    __syncwarp();
    if (lane < nl)
      for (int e = 0; e < ne; e++) t[lane][e] = pull_forward<T, K>(pc, c0 + e, t[lane][e], win);
    __syncwarp();
    if (lane < ne) {
#pragma unroll 8
      for (int r = 0; r < nl; r++) d[(long)r * sx + c0 + lane] = t[r][lane];
    }
    __syncwarp();
  }
  win[0] = win[1] = win[2] = T(0);
  for (int c0 = ((n - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
    const int ne = min(32, n - c0);
    if (lane < ne) {
#pragma unroll 8
      for (int r = 0; r < nl; r++) t[r][lane] = d[(long)r * sx + c0 + lane];
    }
    __syncwarp();
    if (lane < nl)
      for (int e = ne - 1; e >= 0; e--) t[lane][e] = pull_backward<T, K>(pc, c0 + e, t[lane][e], win);
    __syncwarp();
    if (lane < ne) {
#pragma unroll 8
      for (int r = 0; r < nl; r++) d[(long)r * sx + c0 + lane] = t[r][lane];
    }
    __syncwarp();
  }
}

}  // namespace cfd2lcs
