// Device-side building blocks shared by the libcfd2lcs_b200 kernels: grid access,
// ghost rules, trilinear stencil, boundary conditions and node tracking.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "grid.h"

namespace cfd2lcs {

// Device error word bits (folded into the library's error latch after each update).
enum : int {
  ERR_NONFINITE_VELOCITY = 1,
  ERR_TRACKING = 2,
  ERR_UNKNOWN_FLAG = 4,
  ERR_SPLINE_RANGE = 8,
  ERR_ASYNC_COPY = 16,  // a shared-memory staging copy did not complete within its wait limit
};

enum { EULER_ = 0, TRAPEZOIDAL_ = 1, RK2_ = 2, RK3_ = 3, RK4_ = 4 };
// INTERP_SPLINE: B-spline of any order per axis; INTERP_SPLINE4: cubic on every axis (3-D grid);
// INTERP_TSE / INTERP_TSE_LIMIT: Taylor series about the tracked node, without / with limiter;
// INTERP_CTSE / INTERP_CTSE_LIMIT: the same on a non-rectilinear grid (least-squares gradients,
// full coordinate arrays), the only interpolators the reference runs there
enum {
  INTERP_NEAREST = 0,
  INTERP_LINEAR = 1,
  INTERP_SPLINE = 2,
  INTERP_SPLINE4 = 3,
  INTERP_TSE = 4,
  INTERP_TSE_LIMIT = 5,
  INTERP_CTSE = 6,
  INTERP_CTSE_LIMIT = 7
};

__host__ __device__ constexpr bool interp_is_spline(int interp) { return interp == INTERP_SPLINE || interp == INTERP_SPLINE4; }
__host__ __device__ constexpr bool interp_is_curv(int interp) { return interp == INTERP_CTSE || interp == INTERP_CTSE_LIMIT; }

template <typename T>
struct DevGrid {
  GridParams<T> P;
  const T *lt[3];        // node coordinate lines, index 0..n+1
  const T *li[3];        // interpolation lines, index 0..n+1
  // RN(1 / (li[a][i+1] - li[a][i])), index 0..n: the LINEAR stencils' fractions (lin_quotient)
  const T *ri[3] = {nullptr, nullptr, nullptr};
  const T *invd[3];      // inverse half spans, see HostGrid::invd
  const int8_t *flag;    // padded bcflag or nullptr
  const T *nrm[3];       // boundary normals (padded) or nullptr
  // non-rectilinear grids (P.curv), else nullptr:
  const T *X[3] = {nullptr, nullptr, nullptr};      // padded node coordinates
  const T *lsw = nullptr;                           // least-squares weights: plane nb*3 + c holds face
                                                    // neighbour nb's weight in d/dx_c
  const T *pnrm[3] = {nullptr, nullptr, nullptr};   // 2-D grids: unit normal of the data plane per interior node
  const T *invdp[3] = {nullptr, nullptr, nullptr};  // padded inverse half spans
};

template <typename T>
struct FieldPtrs {
  const T *f[3];
};

template <typename T>
struct FieldPtrsW {
  T *f[3];
};

// Forward particles (one per lcs node): position, unwrapped displacement and tracked node
// (the reference's lp%xp, lp%dx, lp%no_scfd).  Storage slot s holds the particle that started
// at interior node id[s]; slot[q] is the inverse map.  The engine re-sorts the slots by grid
// cell during an update, so that a block's particles gather neighbouring spline taps.
template <typename T>
struct Particles {
  T *x[3];
  T *dx[3];
  int *no[3];
  int *id;
  int *slot;
};

__device__ __forceinline__ int pidx(const int sx, const int sxy, int i, int j, int k) { return i + sx * j + sxy * k; }

template <typename T>
__device__ __forceinline__ T clamp01(T v) {
  // max(min(v,1),0) of the reference; a NaN argument yields the bound as gfortran does
  return fmax(fmin(v, T(1)), T(0));
}

// ---------------------------------------------------------------------------------------
// Ghost fill of a padded field, written by the interior node that is the source of each
// ghost cell.  The rules restate exchange_sdata (one rank: periodic SELF copies,
// src/comms_m.f90:679-869) followed by
//   VEL: set_velocity_bc, src/sgrid_m.f90:810-866
//   FM : set_flowmap_bc,  src/flowmap_m.f90:325-392
// vpre: value the periodic copy sees (before interior boundary zeroing); vfin: final
// interior value (what a zero-gradient ghost copies).
// ---------------------------------------------------------------------------------------
enum { GHOST_VEL = 0, GHOST_FM = 1 };

__device__ __forceinline__ int ghost_rule(int kind, int f) {
  // 0: periodic image, 1: zero, 2: copy of the nearest interior node, 3: unknown flag
  if (f == LCS_INTERNAL) return 0;
  if (kind == GHOST_VEL) {
    if (f == LCS_MASK || f == LCS_WALL) return 1;
    if (f == LCS_SLIP || f == LCS_INFLOW || f == LCS_OUTFLOW || f == LCS_2D) return 2;
  } else {
    if (f == LCS_WALL || f == LCS_MASK || f == LCS_INFLOW || f == LCS_OUTFLOW) return 1;
    if (f == LCS_SLIP || f == LCS_2D) return 2;
  }
  return 3;
}

// Every ghost cell has exactly one source node: its periodic image (rule 0) or its
// nearest interior node (rules 1, 2).  The node (i,j,k) enumerates both candidate sets
// and writes the cells whose rule points back at it, so no two threads write one cell.
template <typename T, bool HAS_FLAGS, int KIND, typename TF = T>
__device__ void write_ghosts(const DevGrid<T> &g, TF *const f[3], int i, int j, int k, const TF vpre[3], const TF vfin[3],
                             int *err) {
  const int idx[3] = {i, j, k};
  bool edge = false;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (idx[a] == 1 || idx[a] == g.P.n[a]) edge = true;
  if (!edge) return;
  // clamp side: index 0 next to node 1, n+1 next to node n (rules 1 and 2)
  if (HAS_FLAGS) {
    int ca[3][3], nc[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int n = g.P.n[a], v = idx[a];
      nc[a] = 0;
      ca[a][nc[a]++] = v;
      if (v == 1) ca[a][nc[a]++] = 0;
      if (v == n) ca[a][nc[a]++] = n + 1;
    }
    for (int c2 = 0; c2 < nc[2]; c2++)
      for (int c1 = 0; c1 < nc[1]; c1++)
        for (int c0 = 0; c0 < nc[0]; c0++) {
          if (c0 == 0 && c1 == 0 && c2 == 0) continue;
          const int p = pidx(g.P.sx, g.P.sxy, ca[0][c0], ca[1][c1], ca[2][c2]);
          const int rule = ghost_rule(KIND, (int)g.flag[p]);
          if (rule == 0) continue;
          if (rule == 3) {
            atomicOr(err, ERR_UNKNOWN_FLAG);
            continue;
          }
#pragma unroll
          for (int c = 0; c < 3; c++) f[c][p] = rule == 1 ? TF(0) : vfin[c];
        }
  }
  // wrap side: index n+1 is the image of node 1 and index 0 of node n (rule 0)
  int cw[3][2], nw[3];
  bool any = false;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int n = g.P.n[a], v = idx[a];
    nw[a] = 0;
    cw[a][nw[a]++] = v;
    if (g.P.per[a]) {
      if (v == 1) {
        cw[a][nw[a]++] = n + 1;
        any = true;
      } else if (v == n) {
        cw[a][nw[a]++] = 0;
        any = true;
      }
    }
  }
  if (!any) return;
  for (int c2 = 0; c2 < nw[2]; c2++)
    for (int c1 = 0; c1 < nw[1]; c1++)
      for (int c0 = 0; c0 < nw[0]; c0++) {
        if (c0 == 0 && c1 == 0 && c2 == 0) continue;
        const int p = pidx(g.P.sx, g.P.sxy, cw[0][c0], cw[1][c1], cw[2][c2]);
        if (HAS_FLAGS && ghost_rule(KIND, (int)g.flag[p]) != 0) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) f[c][p] = vpre[c];
      }
}

}  // namespace cfd2lcs
