// __global__ kernels of libcfd2lcs_b200.  One thread per grid node or per particle; the
// fields are ghost-padded SoA arrays (src/structured_m.f90:73-96 layout, i fastest).
#pragma once

#include <cfloat>

#include "advect.cuh"
#include "eig3.h"

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
  if (g.P.curv) return __ldg(g.invdp[a] + pidx(g.P.sx, g.P.sxy, i, j, k));  // per node
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
// Resident blocks of 256 threads per SM asked of the compiler for the two advection kernels,
// i.e. a register cap of 65536 / (256 * blocks).  Without a cap ptxas gives the FP64 RK3 B-spline
// kernels 104 registers (2 blocks, 16 warps per SM); a minimum of 1 block lets it take up to
// 255.  Measured on B200 (ABC 256^3 RK3 CUBIC, turbulence 512^3 RK2 LINEAR): 4 blocks (64
// registers) for the B-spline kernels took the FP64 backward subcycle from 5.02 to 4.32 ms and
// the forward one from 8.85 to 7.52 ms despite a few spilled registers.  The LINEAR backward
// kernel (latency-bound: three dependent gathers per point) with 3 / 4 / 5 blocks: ABC 256^3
// RK2 0.848 / 0.742 / 0.800 ms, turbulence 512^3 8.06 / 7.58 / 7.56 ms (6 blocks, 40
// registers, was 7 % slower than 5 on the turbulence).
#ifndef CFD2LCS_SL_MINB_LINEAR
#define CFD2LCS_SL_MINB_LINEAR 4
#endif
#ifndef CFD2LCS_SL_MINB_SPLINE
#define CFD2LCS_SL_MINB_SPLINE 4
#endif
#ifndef CFD2LCS_FWD_MINB_LINEAR
#define CFD2LCS_FWD_MINB_LINEAR 4
#endif
#ifndef CFD2LCS_FWD_MINB_SPLINE
#define CFD2LCS_FWD_MINB_SPLINE 4
#endif
template <int INTERP>
constexpr int sl_min_blocks() {
  return interp_is_spline(INTERP) ? CFD2LCS_SL_MINB_SPLINE : CFD2LCS_SL_MINB_LINEAR;
}
template <int INTERP>
constexpr int fwd_min_blocks() {
  return interp_is_spline(INTERP) ? CFD2LCS_FWD_MINB_SPLINE : CFD2LCS_FWD_MINB_LINEAR;
}

template <typename T, typename TV, int INTEG, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256, sl_min_blocks<INTERP>()) k_sl_subcycle(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, FieldPtrs<T> fmo,
                                                      FieldPtrsW<T> fmn, StageTimes S, T dt, int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
  constexpr bool CURV = interp_is_curv(INTERP);
  T x0[3];
  node_xyz<T, CURV>(g, i, j, k, x0);
  int no[3] = {i, j, k};
  T x[3];
  integrate<T, TV, INTEG, INTERP, true>(g, sa, V, S, dt, x0, no, x);
  project_plane<T, CURV>(g, no, x);
  const bool stick = particle_bc<T, HAS_FLAGS, CURV>(g, no, x, err);
  if (stick) {
    x[0] = x0[0];
    x[1] = x0[1];
    x[2] = x0[2];
  }
  T fmp[3];
  const int nod[3] = {i, j, k};
  sample_field<T, INTERP, uniform_basis<T, TV>()>(g, sa, fmo.f, x, nod, fmp);
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
// Refined lcs grids (resolution /= 0, new_sgrid_from_sgrid, src/sgrid_m.f90:446-761): the
// flow map lives on the lcs grid gl, the velocity on the solver grid gs.
//
// k_track_lcs_nodes: each lcs node's solver-grid node (init_lp / reset_lp, src/lp_m.f90:
// 72-90, 261-280: the guess nint(real(i*ni_s)/real(ni_l)) in single precision, then the
// recursive 27-neighbour search of track_lp2node on gs, with the periodic wrap of
// exchange_lpdata for forward sets only), and the position after that tracking.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_track_lcs_nodes(DevGrid<T> gs, DevGrid<T> gl, FieldPtrsW<T> pos, int *no0, int *no1, int *no2,
                                                         int fwd, int *err) {
  int i, j, k;
  if (!node_of_thread(gl.P.n, i, j, k)) return;
  const int q = interior_index(gl.P.n, i, j, k);
  T x[3] = {__ldg(gl.lt[0] + i), __ldg(gl.lt[1] + j), __ldg(gl.lt[2] + k)};
  const int nd[3] = {i, j, k};
  int no[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float r = (float)(nd[a] * gs.P.n[a]) / (float)gl.P.n[a];
    no[a] = min(max((int)roundf(r), 1), gs.P.n[a]);  // nint: half away from zero
  }
  int passes = 0;
  while (true) {
    const bool moved = track_pass(gs, x, no);
    passes++;
    if (passes > gs.P.maxtrack) {
      atomicOr(err, ERR_TRACKING);
      break;
    }
    if (fwd) wrap_particle(gs, x, no);
    if (!moved) break;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) pos.f[c][q] = x[c];
  no0[q] = no[0];
  no1[q] = no[1];
  no2[q] = no[2];
}

// One backward SL subcycle on a refined lcs grid (update_flowmap_sl, src/flowmap_m.f90:17-104,
// with lp%sgrid /= scfd%sgrid): the stages integrate from the node's tracked position with
// the velocity on gs around its solver node (set_lp_bc clamps that node in place, so the
// clamped node is written back and used by later subcycles, as lp%no_scfd is), the previous
// flow map is sampled on gl around the lcs node, the mask comes from the solver node's flag
// and the flow-map boundary rule from the lcs node's.  B-spline interpolation samples the
// velocity blends with the solver grid's axes sas and the flow-map coefficients with the lcs
// grid's axes sal.
template <typename T, typename TV, int INTEG, int INTERP, bool FS, bool FL>
__global__ void __launch_bounds__(256) k_sl_refined(DevGrid<T> gl, DevGrid<T> gs, SplineAxes<T> sas, SplineAxes<T> sal, FieldPtrs<T> pos,
                                                    int *no0, int *no1, int *no2, VelFields<TV> V, FieldPtrs<T> fmo, FieldPtrsW<T> fmn,
                                                    StageTimes S, T dt, int *err) {
  int i, j, k;
  if (!node_of_thread(gl.P.n, i, j, k)) return;
  const int p = pidx(gl.P.sx, gl.P.sxy, i, j, k), q = interior_index(gl.P.n, i, j, k);
  const T x0[3] = {pos.f[0][q], pos.f[1][q], pos.f[2][q]};
  int no[3] = {no0[q], no1[q], no2[q]};
  // the mask is taken before the clamp (update_flowmap_sl sets it before integrating)
  const int fs = FS ? (int)gs.flag[pidx(gs.P.sx, gs.P.sxy, no[0], no[1], no[2])] : (int)LCS_INTERNAL;
  T x[3];
  integrate<T, TV, INTEG, INTERP, false>(gs, sas, V, S, dt, x0, no, x);
  project_plane(gs, no, x);
  const bool stick = particle_bc<T, FS>(gs, no, x, err);
  if (stick) {
    x[0] = x0[0];
    x[1] = x0[1];
    x[2] = x0[2];
  }
  no0[q] = no[0];
  no1[q] = no[1];
  no2[q] = no[2];
  T fmp[3];
  const int nod[3] = {i, j, k};
  sample_field<T, INTERP, uniform_basis<T, TV>()>(gl, sal, fmo.f, x, nod, fmp);
  const T mask = fs != LCS_MASK ? T(1) : T(0);
  const int fl = FL ? (int)gl.flag[p] : (int)LCS_INTERNAL;
  const bool zero = FL && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
  T vpre[3], vfin[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    vpre[c] = (fmp[c] + (x[c] - x0[c])) * mask;
    vfin[c] = zero ? T(0) : vpre[c];
    fmn.f[c][p] = vfin[c];
  }
  write_ghosts<T, FL, GHOST_FM>(gl, fmn.f, i, j, k, vpre, vfin, err);
}

// The velocity snapshot on the padded solver grid as reconstruct_flowmap reads it back
// (src/flowmap_m.f90:214-234): interior values, ghosts copied from their periodic images
// (exchange_sdata with max connectivity: a ghost all of whose out-of-range directions are
// periodic), every other ghost 0 (init_sr1; no velocity boundary rule here).
template <typename T, typename TV>
__global__ void __launch_bounds__(256) k_pad_snapshot(DevGrid<T> g, FieldPtrs<TV> src, FieldPtrsW<TV> dst, long ntot) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntot) return;
  int idx[3] = {(int)(p % g.P.sx), (int)((p / g.P.sx) % (g.P.sxy / g.P.sx)), (int)(p / g.P.sxy)};
  bool ok = true;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int n = g.P.n[a];
    if (idx[a] < 1 || idx[a] > n) {
      if (!g.P.per[a]) ok = false;
      idx[a] = idx[a] < 1 ? idx[a] + n : idx[a] - n;
    }
  }
  const int q = ok ? interior_index(g.P.n, idx[0], idx[1], idx[2]) : 0;
#pragma unroll
  for (int c = 0; c < 3; c++) dst.f[c][p] = ok ? src.f[c][q] : TV(0);
}

// lp%ugrid of a refined lcs grid: the padded snapshot (V: its values as un = unp1, or its
// spline coefficients as the stage-0 blend) sampled with the interpolator at every lcs node,
// around the node reset_lp guesses (nint(real(i*ni_s)/real(ni_l)), not tracked).
template <typename T, typename TV, int INTERP>
__global__ void __launch_bounds__(256) k_sample_ugrid(DevGrid<T> gl, DevGrid<T> gs, SplineAxes<T> sa, VelFields<TV> V, FieldPtrsW<T> out) {
  int i, j, k;
  if (!node_of_thread(gl.P.n, i, j, k)) return;
  const int q = interior_index(gl.P.n, i, j, k);
  const T x[3] = {__ldg(gl.lt[0] + i), __ldg(gl.lt[1] + j), __ldg(gl.lt[2] + k)};
  const int nd[3] = {i, j, k};
  int no[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float r = (float)(nd[a] * gs.P.n[a]) / (float)gl.P.n[a];
    no[a] = min(max((int)roundf(r), 1), gs.P.n[a]);
  }
  T u[3];
  sample_velocity<T, TV, INTERP>(gs, sa, V, x, no, T(0), 0, u);
#pragma unroll
  for (int c = 0; c < 3; c++) out.f[c][q] = u[c];
}

// Forward particles back to the lcs nodes (reset_lp + track_lp2node on the solver grid): the
// positions and solver nodes k_track_lcs_nodes found, in node order.
template <typename T>
__global__ void __launch_bounds__(256) k_reset_refined(DevGrid<T> gl, FieldPtrs<T> pos, const int *no0, const int *no1, const int *no2,
                                                       Particles<T> P) {
  int i, j, k;
  if (!node_of_thread(gl.P.n, i, j, k)) return;
  const int q = interior_index(gl.P.n, i, j, k);
  const int nd[3] = {no0[q], no1[q], no2[q]};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    P.x[c][q] = pos.f[c][q];
    P.dx[c][q] = T(0);
    P.no[c][q] = nd[c];
  }
  P.id[q] = q;
  P.slot[q] = q;
}

// ---------------------------------------------------------------------------------------
// K6  one forward particle subcycle (update_lp, src/lp_motion_m.f90:15-54): integrate,
// project, BC, stick, accumulate the displacement, one pass of the node search and the
// periodic wrap of exchange_lpdata.  Thread q advances the particle in storage slot q.
// ---------------------------------------------------------------------------------------
template <typename T, typename TV, int INTEG, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256, fwd_min_blocks<INTERP>()) k_fwd_subcycle(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, Particles<T> P, StageTimes S,
                                                       T dt, int np, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  T xn[3] = {P.x[0][q], P.x[1][q], P.x[2][q]};
  int no[3] = {P.no[0][q], P.no[1][q], P.no[2][q]};
  // the accumulated displacement is read up front, off the integration's dependent chain
  const T dx0[3] = {P.dx[0][q], P.dx[1][q], P.dx[2][q]};
  constexpr bool CURV = interp_is_curv(INTERP);
  T x[3];
  integrate<T, TV, INTEG, INTERP, false, particle_uniform_basis()>(g, sa, V, S, dt, xn, no, x);
  project_plane<T, CURV>(g, no, x);
  const bool stick = particle_bc<T, HAS_FLAGS, CURV>(g, no, x, err);
  if (stick) {
    x[0] = xn[0];
    x[1] = xn[1];
    x[2] = xn[2];
  }
#pragma unroll
  for (int c = 0; c < 3; c++) P.dx[c][q] = dx0[c] + (x[c] - xn[c]);
  track_pass<T, CURV>(g, x, no);
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
    const int q = P.slot[interior_index(g.P.n, i, j, k)];
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
// On a non-rectilinear grid (CURV) the node guess is comms_m.f90:1662-1673's: per direction a,
// nint((imin_x + imin_y + imin_z)/3) + nint((s dx_a + t dy_a + u dz_a)/3) from the index
// positions of the coordinate extremes (GridParams::guess0, guessd).
template <typename T, bool CURV = false>
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
  if constexpr (CURV) {
    T st[3];
#pragma unroll
    for (int a = 0; a < 3; a++) st[a] = clamp01((x[a] - bb[a]) / (bb[a + 3] - bb[a]));
    const T third = T(1) / T(3);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const T sum = add_rn(add_rn(mul_rn(st[0], g.P.guessd[a][0]), mul_rn(st[1], g.P.guessd[a][1])), mul_rn(st[2], g.P.guessd[a][2]));
      const int v = g.P.guess0[a] + (int)round(mul_rn(third, sum));
      no[a] = min(max(v, 1), g.P.n[a]);
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const T s = clamp01((x[a] - bb[a]) / (bb[a + 3] - bb[a]));
      const int v = (int)round(T(g.P.n[a]) * s);  // nint(real(n)*s): half away from zero
      no[a] = min(max(v, 1), g.P.n[a]);
    }
  }
}

template <typename T, int INTERP, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_compose(DevGrid<T> g, SplineAxes<T> sa, const T *const *slots, int nsl, FieldPtrsW<T> out,
                                                  int *err) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  constexpr bool CURV = interp_is_curv(INTERP);
  T x[3];
  node_xyz<T, CURV>(g, i, j, k, x);
  int no[3] = {i, j, k};
  T d[3] = {T(0), T(0), T(0)};
  for (int m = 0; m < nsl; m++) {
    const T *const f[3] = {slots[3 * m], slots[3 * m + 1], slots[3 * m + 2]};
    project_plane<T, CURV>(g, no, x);
    particle_bc<T, HAS_FLAGS, CURV>(g, no, x, err);
    T up[3];
    sample_field<T, INTERP, particle_uniform_basis()>(g, sa, f, x, no, up);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[c] = x[c] + up[c];
      d[c] = d[c] + up[c];
    }
    alltoall_wrap<T, CURV>(g, x, no);
    int passes = 0;
    while (true) {
      const bool moved = track_pass<T, CURV>(g, x, no);
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

// K4 one sub-flow map at a time, for large grids: the composition particles (one per lcs node:
// position P.x, accumulated displacement P.dx, tracked node P.no, origin node P.id) are
// re-sorted by cell between sub-maps (k_particle_count / k_particle_scatter), so the warps of
// one step gather neighbouring taps -- after a few sub-maps the particles of neighbouring nodes
// are far apart and the node-ordered k_compose gathers each tap sector from HBM.  The per-point
// sequence is k_compose's loop body, the state kept exactly between steps, so the composed map
// is bitwise k_compose's.  k_reset_particles starts the particles at their nodes.
// MINB: resident blocks of 256 threads per SM asked of the compiler (register cap 65536 / (256 MINB))
template <typename T, int INTERP, bool HAS_FLAGS, int MINB = 2>
__global__ void __launch_bounds__(256, MINB) k_compose_step(DevGrid<T> g, SplineAxes<T> sa, FieldPtrs<T> f, Particles<T> P, int np, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  T x[3] = {P.x[0][q], P.x[1][q], P.x[2][q]};
  int no[3] = {P.no[0][q], P.no[1][q], P.no[2][q]};
  T d[3] = {P.dx[0][q], P.dx[1][q], P.dx[2][q]};
  constexpr bool CURV = interp_is_curv(INTERP);
  project_plane<T, CURV>(g, no, x);
  particle_bc<T, HAS_FLAGS, CURV>(g, no, x, err);
  T up[3];
  sample_field<T, INTERP, particle_uniform_basis()>(g, sa, f.f, x, no, up);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    x[c] = x[c] + up[c];
    d[c] = d[c] + up[c];
  }
  alltoall_wrap<T, CURV>(g, x, no);
  int passes = 0;
  while (true) {
    const bool moved = track_pass<T, CURV>(g, x, no);
    passes++;
    if (passes > g.P.maxtrack) {
      atomicOr(err, ERR_TRACKING);
      break;
    }
    wrap_particle(g, x, no);
    if (!moved) break;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    P.x[c][q] = x[c];
    P.no[c][q] = no[c];
    P.dx[c][q] = d[c];
  }
}

// the composed map in node order (exchange_lpmap), after the interior flow-map BC
template <typename T, bool HAS_FLAGS>
__global__ void __launch_bounds__(256) k_compose_finish(DevGrid<T> g, Particles<T> P, FieldPtrsW<T> out, int np) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const int id = P.id[q];
  bool zero = false;
  if (HAS_FLAGS) {
    const int i = id % g.P.n[0] + 1, j = (id / g.P.n[0]) % g.P.n[1] + 1, k = id / (g.P.n[0] * g.P.n[1]) + 1;
    const int fl = (int)g.flag[pidx(g.P.sx, g.P.sxy, i, j, k)];
    zero = fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) out.f[c][id] = zero ? T(0) : P.dx[c][q];
}

// ---------------------------------------------------------------------------------------
// K5  FTLE (compute_ftle, src/lcs_m.f90:66-193 with grad_sr1, src/gradient_m.f90:11-66):
// central differences of the composed displacement map (face ghosts: periodic image, or
// the flow-map ghost rule), right Cauchy-Green tensor of the displacement gradient in
// FP64, largest eigenvalue in closed form (eig3.h; the reference calls LAPACK DSYEV),
// ftle = log(max(sqrt(lam), tiny))/T.
// ---------------------------------------------------------------------------------------
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

// CURV: a non-rectilinear grid, gradient by grad_sr1_ls (src/lcs_m.f90:129-133): per
// component, the face neighbours' differences (the same ghost values) times the node's
// least-squares weights, summed in NBR_OFFSET order from zero in T.
template <typename T, typename R, bool HAS_FLAGS, bool CURV = false>
__global__ void __launch_bounds__(256) k_ftle(DevGrid<T> g, FieldPtrs<T> fm, R *__restrict__ ftle, R Tint, int incompressible) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  double G[3][3];  // G[c][a] = d fm_c / d x_a
  if (CURV) {
    const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
    const size_t plane = (size_t)g.P.sxy * (g.P.n[2] + 2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T f0 = __ldg(fm.f[c] + interior_index(g.P.n, i, j, k));
      T gr[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int nb = 0; nb < 6; nb++) {
        const T df = fm_neighbour<T, R, HAS_FLAGS>(g, fm.f[c], nb % 3, i, j, k, nb < 3 ? -1 : 1) - f0;
#pragma unroll
        for (int a = 0; a < 3; a++) gr[a] = add_rn(gr[a], mul_rn(df, __ldg(g.lsw + (size_t)(nb * 3 + a) * plane + p)));
      }
#pragma unroll
      for (int a = 0; a < 3; a++) G[c][a] = (double)gr[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 3 && !CURV; a++) {
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
  const double lam = eig3_max_closed(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
  const R sq = sqrt((R)lam);
  const R tiny = sizeof(R) == 8 ? (R)DBL_MIN : (R)FLT_MIN;
  const R mx = sq > tiny ? sq : tiny;  // max(sqrt(W3), tiny): NaN yields tiny
  R v = log(mx) / Tint;
  if (incompressible) v = v > R(0) ? v : R(0);
  ftle[interior_index(g.P.n, i, j, k)] = v;
}

// FTLE with AUX_GRID (compute_ftle, src/lcs_m.f90:95-127): the displacement gradient from the
// composed maps of the six auxiliary particle sets, d fm_c / d x_a = (fm_c[a+ side] - fm_c[a-
// side]) / den_a, den_a the separation of the two auxiliary nodes (left 0 where it is not
// above 100 tiny); then the same Cauchy-Green, eigenvalue and log as k_ftle.
template <typename T>
struct AuxMaps {
  const T *lo[3][3];  // [axis][component]: composed maps of the X0, Y0, Z0 sets (interior)
  const T *hi[3][3];  // X1, Y1, Z1
  const T *den[3];    // per node separation along each axis
};

template <typename T, typename R>
__global__ void __launch_bounds__(256) k_ftle_aux(DevGrid<T> g, const __grid_constant__ AuxMaps<T> M, R *__restrict__ ftle, R Tint,
                                                  int incompressible) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int q = interior_index(g.P.n, i, j, k);
  const T small = T(100) * (sizeof(T) == 8 ? (T)DBL_MIN : (T)FLT_MIN);
  double G[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const T den = M.den[a][q];
#pragma unroll
    for (int c = 0; c < 3; c++) G[c][a] = fabs(den) > small ? (double)((M.hi[a][c][q] - M.lo[a][c][q]) / den) : 0.0;
  }
  double C[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) C[a][b] = G[0][a] * G[0][b] + G[1][a] * G[1][b] + G[2][a] * G[2][b];
  const double lam = eig3_max_closed(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
  const R sq = sqrt((R)lam);
  const R tiny = sizeof(R) == 8 ? (R)DBL_MIN : (R)FLT_MIN;
  const R mx = sq > tiny ? sq : tiny;
  R v = log(mx) / Tint;
  if (incompressible) v = v > R(0) ? v : R(0);
  ftle[q] = v;
}

// ---------------------------------------------------------------------------------------
// Velocity invariants (compute_invariants, src/invariants_m.f90:15-208) of one frame from
// the velocity snapshot of the reconstruction's starting step (nodal values, interior
// arrays; null: no snapshot, the zeroed lp%ugrid of the reference).  Gradient by central
// differences with face neighbours: periodic images, zero ghosts elsewhere (grad_sr1,
// src/gradient_m.f90:11-66, after exchange_sdata of the never-bounded ugrid).  Outputs the
// Q, D, C fields (out) and H, lambda-2 (out2) in the reference's expressions and order.
// ---------------------------------------------------------------------------------------
// all three eigenvalues (ascending) of a symmetric 3x3, cyclic Jacobi in FP64
__device__ __forceinline__ void eig3_all(double a00, double a01, double a02, double a11, double a12, double a22, double w[3]) {
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
  double x = a[0][0], y = a[1][1], z = a[2][2], t;
  if (y < x) { t = y; y = x; x = t; }
  if (z < y) { t = z; z = y; y = t; }
  if (y < x) { t = y; y = x; x = t; }
  w[0] = x;
  w[1] = y;
  w[2] = z;
}

template <typename T, typename TU>
__device__ __forceinline__ T ugrid_neighbour(const DevGrid<T> &g, const TU *__restrict__ f, int a, int i, int j, int k, int step) {
  int idx[3] = {i, j, k};
  idx[a] += step;
  const int n = g.P.n[a];
  if (idx[a] < 1 || idx[a] > n) {
    if (!g.P.per[a]) return T(0);
    idx[a] = idx[a] < 1 ? idx[a] + n : idx[a] - n;
  }
  return T(__ldg(f + interior_index(g.P.n, idx[0], idx[1], idx[2])));
}

// CURV: a non-rectilinear grid, gradient by grad_sr1_ls (src/invariants_m.f90:38-42) over the
// same face-neighbour values.
template <typename T, typename TU, bool CURV = false>
__global__ void __launch_bounds__(256) k_invariants(DevGrid<T> g, FieldPtrs<TU> u, int have, FieldPtrsW<T> out, FieldPtrsW<T> out2) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  T G[3][3];  // G[c][a] = d u_c / d x_a
  if (CURV) {
    const int p = pidx(g.P.sx, g.P.sxy, i, j, k);
    const size_t plane = (size_t)g.P.sxy * (g.P.n[2] + 2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T f0 = have ? T(__ldg(u.f[c] + interior_index(g.P.n, i, j, k))) : T(0);
#pragma unroll
      for (int a = 0; a < 3; a++) G[c][a] = T(0);
#pragma unroll
      for (int nb = 0; nb < 6; nb++) {
        const T df = (have ? ugrid_neighbour<T, TU>(g, u.f[c], nb % 3, i, j, k, nb < 3 ? -1 : 1) : T(0)) - f0;
#pragma unroll
        for (int a = 0; a < 3; a++) G[c][a] = add_rn(G[c][a], mul_rn(df, __ldg(g.lsw + (size_t)(nb * 3 + a) * plane + p)));
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3 && !CURV; a++) {
    const int idx[3] = {i, j, k};
    const T den = __ldg(g.lt[a] + idx[a] + 1) - __ldg(g.lt[a] + idx[a] - 1);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T fp = have ? ugrid_neighbour<T, TU>(g, u.f[c], a, i, j, k, +1) : T(0);
      const T fq = have ? ugrid_neighbour<T, TU>(g, u.f[c], a, i, j, k, -1) : T(0);
      G[c][a] = g.P.n[a] == 1 ? T(0) : (fp - fq) / den;
    }
  }
  const T d1u1 = G[0][0], d2u1 = G[0][1], d3u1 = G[0][2];
  const T d1u2 = G[1][0], d2u2 = G[1][1], d3u2 = G[1][2];
  const T d1u3 = G[2][0], d2u3 = G[2][1], d3u3 = G[2][2];
  const T S11 = d1u1 + d1u1, S12 = d1u2 + d2u1, S13 = d1u3 + d3u1;
  const T S21 = d2u1 + d1u2, S22 = d2u2 + d2u2, S23 = d2u3 + d3u2;
  const T S31 = d3u1 + d1u3, S32 = d3u2 + d2u3, S33 = d3u3 + d3u3;
  const T W11 = d1u1 - d1u1, W12 = d1u2 - d2u1, W13 = d1u3 - d3u1;
  const T W21 = d2u1 - d1u2, W22 = d2u2 - d2u2, W23 = d2u3 - d3u2;
  const T W31 = d3u1 - d1u3, W32 = d3u2 - d2u3, W33 = d3u3 - d3u3;
  const T eigth = T(1. / 8.), twenyforth = T(1. / 24.), coef = T(27. / 4.);
  T INV[5];
  INV[0] = -eigth * (S11 * S11 + S12 * S21 + S13 * S31 + S21 * S12 + S22 * S22 + S23 * S32 + S31 * S13 + S32 * S23 + S33 * S33);
  INV[1] = -twenyforth * (S11 * S11 * S11 + S11 * S12 * S21 + S11 * S13 * S31 + S21 * S11 * S12 + S21 * S12 * S22 + S21 * S13 * S32 +
                          S31 * S11 * S13 + S31 * S12 * S23 + S31 * S13 * S33 + S12 * S21 * S11 + S12 * S22 * S21 + S12 * S23 * S31 +
                          S13 * S31 * S11 + S13 * S32 * S21 + S13 * S33 * S31 + S22 * S22 * S22 + S22 * S21 * S12 + S22 * S23 * S32 +
                          S23 * S31 * S13 + S23 * S32 * S22 + S23 * S33 * S32 + S32 * S22 * S23 + S32 * S21 * S13 + S32 * S23 * S33 +
                          S33 * S33 * S33 + S33 * S23 * S32 + S33 * S13 * S31);
  INV[2] = INV[0] - eigth * (W11 * W11 + W12 * W21 + W13 * W31 + W21 * W12 + W22 * W22 + W23 * W32 + W31 * W13 + W32 * W23 + W33 * W33);
  INV[3] = INV[1] - eigth * (W11 * W11 * S11 + W11 * W12 * S21 + W11 * W13 * S31 + W21 * W11 * S12 + W21 * W12 * S22 + W21 * W13 * S32 +
                             W31 * W11 * S13 + W31 * W12 * S23 + W31 * W13 * S33 + W12 * W21 * S11 + W12 * W22 * S21 + W12 * W23 * S31 +
                             W13 * W31 * S11 + W13 * W32 * S21 + W13 * W33 * S31 + W22 * W22 * S22 + W22 * W21 * S12 + W22 * W23 * S32 +
                             W23 * W31 * S13 + W23 * W32 * S22 + W23 * W33 * S32 + W32 * W22 * S23 + W32 * W21 * S13 + W32 * W23 * S33 +
                             W33 * W33 * S33 + W33 * W23 * S32 + W33 * W13 * S31);
  INV[4] = INV[2] - INV[0];
  const int q = interior_index(g.P.n, i, j, k);
  out.f[0][q] = INV[2] > T(0) ? T(1) : T(0);
  const T D = INV[2] * INV[2] * INV[2] + coef * INV[3] * INV[3];
  out.f[1][q] = (D > T(0) && INV[3] > T(0)) ? T(1) : (D > T(0) ? T(2) : (INV[3] > T(0) ? T(3) : T(4)));
  out.f[2][q] = INV[1] > T(0) ? T(1) : T(0);
  out2.f[0][q] = sqrt(-INV[4] / INV[0]);
  // S^2 + Omega^2 (upper triangle, third diagonal entry 0 as the reference sets it), with
  // rounded products so that no multiply-add contraction moves a middle eigenvalue that sits
  // at zero (A(3,3) = 0 makes exact zeros common) across the sign test
  auto dot6 = [](T a0, T b0, T a1, T b1, T a2, T b2, T a3, T b3, T a4, T b4, T a5, T b5) {
    return mul_rn(a0, b0) + mul_rn(a1, b1) + mul_rn(a2, b2) + mul_rn(a3, b3) + mul_rn(a4, b4) + mul_rn(a5, b5);
  };
  double w[3];
  eig3_all((double)dot6(S11, S11, S21, S12, S31, S13, W11, W11, W21, W12, W31, W13),
           (double)dot6(S12, S11, S22, S12, S32, S13, W12, W11, W22, W12, W32, W13),
           (double)dot6(S13, S11, S23, S12, S33, S13, W13, W11, W23, W12, W33, W13),
           (double)dot6(S12, S21, S22, S22, S32, S23, W12, W21, W22, W22, W32, W23),
           (double)dot6(S13, S21, S23, S22, S33, S23, W13, W21, W23, W22, W33, W23), 0.0, w);
  out2.f[1][q] = w[1] < 0.0 ? T(1) : T(0);
}

// velocity snapshot of the ring: interior of the padded level, in the storage type
template <typename T, typename TV>
__global__ void __launch_bounds__(256) k_vel_snapshot(DevGrid<T> g, FieldPtrs<TV> u, FieldPtrsW<TV> dst) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int p = pidx(g.P.sx, g.P.sxy, i, j, k), q = interior_index(g.P.n, i, j, k);
#pragma unroll
  for (int c = 0; c < 3; c++) dst.f[c][q] = u.f[c][p];
}

// Reset of forward particles to their grid nodes (reset_lp, src/lp_m.f90:228-294), in node
// order.
template <typename T>
__global__ void k_reset_particles(DevGrid<T> g, Particles<T> P) {
  int i, j, k;
  if (!node_of_thread(g.P.n, i, j, k)) return;
  const int q = interior_index(g.P.n, i, j, k);
  const int nd[3] = {i, j, k};
  T x[3];
  if (g.P.curv) node_xyz<T, true>(g, i, j, k, x);
  else node_xyz<T, false>(g, i, j, k, x);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    P.x[c][q] = x[c];
    P.dx[c][q] = T(0);
    P.no[c][q] = nd[c];
  }
  P.id[q] = q;
  P.slot[q] = q;
}

// ---------------------------------------------------------------------------------------
// Counting sort of the forward particle slots by grid cell: tiles of 32 (x) x 4 (y) x 2 (z)
// cells, x fastest inside a tile.  A block of 256 particles then covers about one such tile,
// so its warps share the y and z spline rows the way the backward kernel's blocks do (L1
// reuse across the block), and each warp walks along x.  Measured on B200 (ABC 256^3 CUBIC,
// forward launch): tiles 32 x 8 x 1 / 32 x 4 x 2 / 32 x 2 x 4 took 6.91 / 6.72 / 6.82 ms (FP64
// velocity) and 4.20 / 4.06 / 4.12 ms (FP32).  Steps: count per cell key, exclusive scan of the counts in chunks of
// SORT_TILE, and a scatter that moves every particle to its key's next free slot.  Particles
// of one cell land in arbitrary order, which no result depends on.  The count array returns
// to zero inside the scan, ready for the next sort.
// ---------------------------------------------------------------------------------------
constexpr int SORT_TILE = 2048;  // 256 threads x 8 counts

// Cell tiles of the order: tx x ty x tz cells (tx ty tz = 256), x fastest inside a tile and
// tiles in x, y, z order; cells c_a in 0..n_a per axis, padded to whole tiles.  The gathering
// forward kernel takes 32 x 4 x 2 (32 x 8/SORT_TZ x SORT_TZ; measured on B200, see the engine),
// the staged forward kernel 16 x 4 x 4 (its shared-memory box is that tile widened by 4 cells).
#ifndef CFD2LCS_SORT_TZ
#define CFD2LCS_SORT_TZ 2
#endif
constexpr int SORT_TZ = CFD2LCS_SORT_TZ, SORT_TY = 8 / SORT_TZ;

struct SortTiles {
  int tx, ty, tz;     // cells per tile along each axis
  int ntx, nty, ntz;  // tiles along each axis
};

__host__ __device__ inline SortTiles sort_tiles(const int n[3], int tx, int ty, int tz) {
  SortTiles s;
  s.tx = tx;
  s.ty = ty;
  s.tz = tz;
  s.ntx = (n[0] + 1 + tx - 1) / tx;
  s.nty = (n[1] + 1 + ty - 1) / ty;
  s.ntz = (n[2] + 1 + tz - 1) / tz;
  return s;
}

__host__ __device__ inline long sort_key_space(const SortTiles &s) { return (long)s.ntz * s.nty * s.ntx * 256; }

// cell c in 0..n along each axis: the tracked node (clamped to the interior), minus one when
// the particle lies below the node's line
template <typename T>
__global__ void __launch_bounds__(256) k_particle_count(DevGrid<T> g, Particles<T> P, unsigned *key, int *cnt, int np, SortTiles st) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  int c[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int v = min(max(P.no[a][s], 1), g.P.n[a]);
    c[a] = v - (P.x[a][s] < __ldg(g.lt[a] + v) ? 1 : 0);
  }
  const unsigned tile = (unsigned)(((c[2] / st.tz) * st.nty + c[1] / st.ty) * st.ntx + c[0] / st.tx);
  const unsigned kq = tile * 256u + (unsigned)(((c[2] % st.tz) * st.ty + c[1] % st.ty) * st.tx + c[0] % st.tx);
  key[s] = kq;
  atomicAdd(cnt + kq, 1);
}

// First slot of sort tile t after k_particle_scatter, which leaves offs[k] at the end of key k's
// slots within its SORT_TILE chunk and tsum[c] at the chunk's first slot; t = the number of
// tiles gives np.
__device__ __forceinline__ int sort_tile_start(const int *offs, const int *tsum, long t, long ntiles, int np) {
  if (t >= ntiles) return np;
  const long k0 = t * 256;
  return __ldg(tsum + k0 / SORT_TILE) + ((k0 % SORT_TILE) ? __ldg(offs + k0 - 1) : 0);
}

// exclusive scan of cnt within each chunk into offs (cnt reset to 0), chunk totals to tsum
static __global__ void __launch_bounds__(256) k_scan_tiles(int *cnt, int *offs, int *tsum, int n) {
  __shared__ int wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long base = (long)blockIdx.x * SORT_TILE + threadIdx.x * 8;
  int v[8], run = 0;
#pragma unroll
  for (int e = 0; e < 8; e++) {
    const long q = base + e;
    const int c = q < n ? cnt[q] : 0;
    v[e] = run;
    run += c;
    if (q < n) cnt[q] = 0;
  }
  int x = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < 8 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < 8) wsum[lane] = w;
  }
  __syncthreads();
  const int excl = x - run + (warp ? wsum[warp - 1] : 0);
#pragma unroll
  for (int e = 0; e < 8; e++)
    if (base + e < n) offs[base + e] = excl + v[e];
  if (threadIdx.x == 255) tsum[blockIdx.x] = excl + run;
}

// exclusive scan of the chunk totals in place (one block)
static __global__ void __launch_bounds__(1024) k_scan_tile_sums(int *tsum, int nt) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nt; b0 += 1024) {
    const int q = b0 + threadIdx.x;
    const int c = q < nt ? tsum[q] : 0;
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const int incl = x + (warp ? wsum[warp - 1] : 0);
    if (q < nt) tsum[q] = carry + incl - c;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
}

// slot of particle s: its key's chunk base + in-chunk offset + arrival order at the key
template <typename T>
__global__ void __launch_bounds__(256) k_particle_scatter(Particles<T> src, Particles<T> dst, const unsigned *__restrict__ key,
                                                           int *offs, const int *__restrict__ tsum, int np) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= np) return;
  const unsigned kq = key[s];
  const int d = __ldg(tsum + kq / SORT_TILE) + atomicAdd(offs + kq, 1);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    dst.x[c][d] = src.x[c][s];
    dst.dx[c][d] = src.dx[c][s];
    dst.no[c][d] = src.no[c][s];
  }
  const int id = src.id[s];
  dst.id[d] = id;
  dst.slot[id] = d;
}

// Time blends of two padded coefficient fields for the RK stages of a subcycle that have no
// blend yet: out_m = (1-ct_m) a + ct_m b for m < nout, so a and b are read once for all of
// them.  Two elements per thread (8- or 16-byte vector accesses), component blockIdx.y.
template <typename T>
struct Pair;
template <>
struct Pair<double> {
  using type = double2;
};
template <>
struct Pair<float> {
  using type = float2;
};

template <typename T>
struct BlendOut {
  T *f[3][3];  // [output][component]
  T omc[3], ct[3];
};

template <typename T>
__global__ void __launch_bounds__(256) k_blend(const __grid_constant__ FieldPtrs<T> a, const __grid_constant__ FieldPtrs<T> b,
                                                const __grid_constant__ BlendOut<T> o, int nout, long ntot) {
  using P2 = typename Pair<T>::type;
  const long h = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int comp = blockIdx.y;
  const long q = 2 * h;
  if (q + 1 < ntot) {
    const P2 va = __ldg(reinterpret_cast<const P2 *>(a.f[comp]) + h);
    const P2 vb = __ldg(reinterpret_cast<const P2 *>(b.f[comp]) + h);
    for (int m = 0; m < nout; m++) {
      P2 r;
      r.x = o.omc[m] * va.x + o.ct[m] * vb.x;
      r.y = o.omc[m] * va.y + o.ct[m] * vb.y;
      reinterpret_cast<P2 *>(o.f[m][comp])[h] = r;
    }
  } else if (q < ntot) {
    const T va = __ldg(a.f[comp] + q), vb = __ldg(b.f[comp] + q);
    for (int m = 0; m < nout; m++) o.f[m][comp][q] = o.omc[m] * va + o.ct[m] * vb;
  }
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
// resident blocks asked of the compiler: measured on B200 (192^3, FP64, K = 4) 2 / 3 / 4 blocks
// took 0.153 / 0.129 / 0.159 ms per launch
#ifndef CFD2LCS_FIT_MINB
#define CFD2LCS_FIT_MINB 3
#endif
template <typename T, int K>
__global__ void __launch_bounds__(256, CFD2LCS_FIT_MINB) k_fit_lines(SplineAxis<T> A, const __grid_constant__ FieldPtrs<T> src,
                                                       const __grid_constant__ FieldPtrsW<T> dst, int nfast, long nlines, long es,
                                                       long so) {
  const long L = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= nlines) return;
  const long off = L % nfast + (L / nfast) * so;
  const T *s = src.f[blockIdx.y] + off;
  T *d = dst.f[blockIdx.y] + off;
  const int n = A.n;
  const T *pc = A.pull;
  constexpr int G = 8;
  T win[3] = {T(0), T(0), T(0)};
  const T *sp = s;
  T *dp = d;
  for (int i0 = 0; i0 < n; i0 += G, sp += G * es, dp += G * es) {
    T v[G];
#pragma unroll
    for (int g = 0; g < G; g++) v[g] = (i0 + g < n) ? sp[g * es] : T(0);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i0 + g < n) v[g] = pull_forward<T, K>(pc, i0 + g, v[g], win);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i0 + g < n) dp[g * es] = v[g];
  }
  win[0] = win[1] = win[2] = T(0);
  dp = d + (long)(n - 1) * es;
  for (int i1 = n - 1; i1 >= 0; i1 -= G, dp -= G * es) {
    T v[G];
#pragma unroll
    for (int g = 0; g < G; g++) v[g] = (i1 - g >= 0) ? dp[-g * es] : T(0);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i1 - g >= 0) v[g] = pull_backward<T, K>(pc, i1 - g, v[g], win);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (i1 - g >= 0) dp[-g * es] = v[g];
  }
}

// asynchronous element copy global -> shared (LDGSTS), completed by cp_async_wait
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// x pass: lines are contiguous.  One warp per 32 lines (consecutive j at one k).  Chunks of
// XFIT_W elements of the 32 lines are staged through two shared tiles per warp: the next
// chunk's rows are copied asynchronously (one coalesced row per copy instruction) while one lane
// per line sweeps the current tile, which then goes back to memory as coalesced row stores.
// Chunks of 16 rather than 32 elements halve the shared memory of a block and double the
// resident warps: measured on B200 at 192^3 (FP64), 0.288 -> 0.268 ms per launch.
#ifndef CFD2LCS_XFIT_W
#define CFD2LCS_XFIT_W 16
#endif
constexpr int XFIT_W = CFD2LCS_XFIT_W;  // elements per staged chunk of a line
template <typename T, int K>
__global__ void __launch_bounds__(128) k_fit_xlines(SplineAxis<T> A, const __grid_constant__ FieldPtrs<T> src,
                                                     const __grid_constant__ FieldPtrsW<T> dst, int ny, int nz, long sx, long sxy) {
  extern __shared__ __align__(16) unsigned char fit_smem[];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  T(*tiles)[32][XFIT_W + 1] = reinterpret_cast<T(*)[32][XFIT_W + 1]>(fit_smem) + 2 * wp;
  const int nbf = (ny + 31) / 32;
  const long gw = (long)blockIdx.x * 4 + wp;
  if (gw >= (long)nbf * nz) return;  // warp-uniform
  const int j0 = (int)(gw % nbf) * 32;
  const int nl = min(32, ny - j0);
  const long base = (long)j0 * sx + (gw / nbf) * sxy;
  const T *s = src.f[blockIdx.y] + base;
  T *d = dst.f[blockIdx.y] + base;
  const int n = A.n, nch = (n + XFIT_W - 1) / XFIT_W;
  const T *pc = A.pull;
  // chunk c of the sweep (forward: c-th from the start, backward: from the end)
  auto chunk0 = [&](int c, bool fwd) { return fwd ? c * XFIT_W : (nch - 1 - c) * XFIT_W; };
  auto issue = [&](const T *from, int c0, T(*t)[XFIT_W + 1]) {
    const int ne = min(XFIT_W, n - c0);
    if (lane < ne)
      for (int r = 0; r < nl; r++) cp_async_elem(&t[r][lane], from + (long)r * sx + c0 + lane);
    cp_async_commit();
  };
  T win[3];
  for (int pass = 0; pass < 2; pass++) {
    const bool fwd = pass == 0;
    const T *from = fwd ? s : d;
    win[0] = win[1] = win[2] = T(0);
    issue(from, chunk0(0, fwd), tiles[0]);
    for (int c = 0; c < nch; c++) {
      T(*t)[XFIT_W + 1] = tiles[c & 1];
      if (c + 1 < nch) {
        issue(from, chunk0(c + 1, fwd), tiles[(c + 1) & 1]);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const int c0 = chunk0(c, fwd), ne = min(XFIT_W, n - c0);
      if (lane < nl) {
        if (fwd) {
          if (ne == XFIT_W) {
#pragma unroll
            for (int e = 0; e < XFIT_W; e++) t[lane][e] = pull_forward<T, K>(pc, c0 + e, t[lane][e], win);
          } else {
            for (int e = 0; e < ne; e++) t[lane][e] = pull_forward<T, K>(pc, c0 + e, t[lane][e], win);
          }
        } else {
          if (ne == XFIT_W) {
#pragma unroll
            for (int e = XFIT_W - 1; e >= 0; e--) t[lane][e] = pull_backward<T, K>(pc, c0 + e, t[lane][e], win);
          } else {
            for (int e = ne - 1; e >= 0; e--) t[lane][e] = pull_backward<T, K>(pc, c0 + e, t[lane][e], win);
          }
        }
      }
      __syncwarp();
      if (lane < ne) {
#pragma unroll 8
        for (int r = 0; r < nl; r++) d[(long)r * sx + c0 + lane] = t[r][lane];
      }
      __syncwarp();
    }
  }
}

}  // namespace cfd2lcs
