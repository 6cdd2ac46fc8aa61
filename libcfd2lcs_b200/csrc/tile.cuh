// Backward semi-Lagrangian subcycle with the B-spline taps staged in shared memory: the
// cubic (every axis order 4) form of k_sl_subcycle, update_flowmap_sl
// (src/flowmap_m.f90:17-104) with integrate_lp (src/lp_motion_m.f90:129-360) and the
// CUBIC branch of interp_s2u_r1 (src/lp_tracking_m.f90:476-524).
//
// Why staging works: the subcycle count keeps sum_a |u_a| dt / delta_a <= CFL_MAX = 0.5
// (set_dt, src/lp_motion_m.f90:90-101), so every RK stage position and the departure point
// lie within one cell of their node per axis, and a point in cell [p, p+1) of the padded
// grid reads the coefficients p-1 .. p+2 of the not-a-knot spline.  A block of 32 x 4 x 4
// nodes therefore reads only the coefficient box of its nodes widened by 2 on every side
// (36 x 8 x 8 per component).  The block copies that box into shared memory once per field
// -- the blend of each off-node stage, then the flow map -- with bulk asynchronous copies
// (cp.async.bulk: the TMA engine, one row of the box per copy, completion on an mbarrier),
// and every point contracts its 64 taps per component from shared memory instead of
// gathering them through L1.  A stencil that leaves the box (a point further than the CFL
// bound, e.g. where a spline overshoots) is read from global memory instead; both paths run
// the same FMA sequence (spline_contract), so the result is bitwise that of k_sl_subcycle.
#pragma once

#include "kernels.cuh"

namespace cfd2lcs {

// ---------------------------------------------------------------------------------------
// mbarrier and bulk-copy primitives (PTX).  No multi-CTA or multi-GPU form is used: every
// copy reads this GPU's global memory into the issuing CTA's own shared memory.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete; gives up after about one second of
// SM clock (2^31 cycles) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > (1LL << 31)) return false;
  return true;
}

// bytes (a multiple of 16) from 16-byte aligned global src to 16-byte aligned shared dst
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// orders this thread's earlier shared-memory accesses before later bulk copies into them
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---------------------------------------------------------------------------------------
// Tile geometry
// ---------------------------------------------------------------------------------------
constexpr int SLT_X = 32, SLT_Y = 4, SLT_Z = 4;  // nodes per block (block of 32 x 4 x 2 threads, 2 nodes each)
constexpr int SLT_HALO = 2;
constexpr int SLT_SX = SLT_X + 2 * SLT_HALO, SLT_SY = SLT_Y + 2 * SLT_HALO, SLT_SZ = SLT_Z + 2 * SLT_HALO;
constexpr int SLT_ROWS = SLT_SY * SLT_SZ;  // rows of the box per component
constexpr int SLT_THREADS = 256;

// Row pitch (elements) of the box in shared memory: a row copy starts at the 16-byte boundary
// at or below its first element, so a row holds up to 16/sizeof - 1 leading extra elements.
template <typename TC>
__host__ __device__ constexpr int slt_pitch() {
  return ((SLT_SX + 2 * (16 / (int)sizeof(TC) - 1)) / (16 / (int)sizeof(TC))) * (16 / (int)sizeof(TC));
}
template <typename TC>
__host__ __device__ constexpr int slt_comp() {
  return SLT_ROWS * slt_pitch<TC>();
}
// shared memory of one staged field (3 components); the flow map's type is the widest
template <typename TC>
__host__ __device__ constexpr size_t slt_field_bytes() {
  return (size_t)3 * slt_comp<TC>() * sizeof(TC);
}

// The staged box of a block: origin (padded indices, may lie outside the array) and the part
// inside the padded array, [lo, hi) per axis.
struct TileBox {
  int xs, ys, zs;
  int xlo, xhi, ylo, yhi, zlo, zhi;
};

// Issues the row copies of one 3-component field into buf; threads 0..3*SLT_ROWS-1 each
// arrive once on bar (with the bytes of their row, or none for a row outside the array).
template <typename TC>
__device__ __forceinline__ void slt_fill(TC *buf, const TC *f0, const TC *f1, const TC *f2, const TileBox &b, int sx, int sxy,
                                         uint64_t *bar, int tid) {
  constexpr int E = 16 / (int)sizeof(TC);
  if (tid >= 3 * SLT_ROWS) return;
  const int c = tid / SLT_ROWS, r = tid - c * SLT_ROWS;
  const TC *const src = c == 0 ? f0 : (c == 1 ? f1 : f2);
  const int y = b.ys + r % SLT_SY, z = b.zs + r / SLT_SY;
  if (y >= b.ylo && y < b.yhi && z >= b.zlo && z < b.zhi && b.xhi > b.xlo) {
    const long e = (long)b.xlo + (long)y * sx + (long)z * sxy;
    const long a = e & ~(long)(E - 1);
    const unsigned bytes = (unsigned)((((e - a) + (b.xhi - b.xlo)) * (long)sizeof(TC) + 15) & ~15L);
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(buf + (size_t)c * slt_comp<TC>() + (size_t)r * slt_pitch<TC>(), src + a, bytes, bar);
  } else {
    mbar_arrive(bar);
  }
}

// true when the stencil's 4 x 4 x 4 coefficients are all in the staged box
__device__ __forceinline__ bool slt_inside(const TileBox &b, const int c0[3]) {
  return c0[0] >= b.xlo && c0[0] + 4 <= b.xhi && c0[1] >= b.ylo && c0[1] + 4 <= b.yhi && c0[2] >= b.zlo && c0[2] + 4 <= b.zhi;
}

// One component from the staged box: coefficient (x, y, z) sits in row (z-zs)*SLT_SY + (y-ys)
// at column x - xlo plus the row's alignment shift ((xlo + y sx + z sxy) mod 16/sizeof).
template <typename T, typename TC>
__device__ __forceinline__ TC slt_apply(const SplineAxes<T> &sa, const SplineStencil<T> &st, const TC *comp, const TileBox &b, int sx,
                                        int sxy) {
  constexpr int E = 16 / (int)sizeof(TC);
  const int gy = st.c0[1] * sx + st.c0[2] * sxy + b.xlo;  // global offset of row (c0y, c0z) at column xlo
  const int rb = ((st.c0[2] - b.zs) * SLT_SY + (st.c0[1] - b.ys)) * slt_pitch<TC>() + (st.c0[0] - b.xlo);
  return spline_contract<T, 4, TC>(sa, st, [&](int c1, int c2, int c0) {
    const int shift = (gy + c1 * sx + c2 * sxy) & (E - 1);
    return comp[rb + (c2 * SLT_SY + c1) * slt_pitch<TC>() + shift + c0];
  });
}

#ifndef CFD2LCS_SLT_MINB
#define CFD2LCS_SLT_MINB 2
#endif

template <typename T, typename TV, int INTEG, bool HAS_FLAGS>
__global__ void __launch_bounds__(SLT_THREADS, CFD2LCS_SLT_MINB)
    k_sl_tile(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, FieldPtrs<T> fmo, FieldPtrsW<T> fmn, StageTimes S, T dt, int *err) {
  extern __shared__ __align__(128) unsigned char slt_smem[];
  __shared__ __align__(8) uint64_t bar;
  constexpr bool UNI = !std::is_same<T, TV>::value;
  constexpr int NOFF = INTEG == RK2_ ? 1 : (INTEG == RK3_ ? 2 : (INTEG == RK4_ ? 3 : 0));  // stages off the node
  const T HALF = T(1) / T(2), THIRD = T(1) / T(3), TWOTHIRD = T(2) / T(3), SIXTH = T(1) / T(6), TWO = T(2);
  const int tid = threadIdx.x + 32 * (threadIdx.y + SLT_Y * threadIdx.z);
  const int sx = g.P.sx, sxy = g.P.sxy;
  TileBox b;
  const int I0 = 1 + (int)blockIdx.x * SLT_X, J0 = 1 + (int)blockIdx.y * SLT_Y, K0 = 1 + (int)blockIdx.z * SLT_Z;
  b.xs = I0 - SLT_HALO;
  b.ys = J0 - SLT_HALO;
  b.zs = K0 - SLT_HALO;
  b.xlo = max(b.xs, 0);
  b.xhi = min(b.xs + SLT_SX, sx);
  b.ylo = max(b.ys, 0);
  b.yhi = min(b.ys + SLT_SY, g.P.n[1] + 2);
  b.zlo = max(b.zs, 0);
  b.zhi = min(b.zs + SLT_SZ, g.P.n[2] + 2);
  TV *const tv = reinterpret_cast<TV *>(slt_smem);
  T *const tf = reinterpret_cast<T *>(slt_smem);
  if (tid == 0) mbar_init(&bar, 3 * SLT_ROWS);
  __syncthreads();
  if (NOFF > 0) slt_fill<TV>(tv, V.cs[1][0], V.cs[1][1], V.cs[1][2], b, sx, sxy, &bar, tid);
  else slt_fill<T>(tf, fmo.f[0], fmo.f[1], fmo.f[2], b, sx, sxy, &bar, tid);

  // the thread's two nodes: (i, j, k) and (i, j, k + 2)
  const int i = I0 + (int)threadIdx.x, j = J0 + (int)threadIdx.y;
  int kq[2] = {K0 + (int)threadIdx.z, K0 + (int)threadIdx.z + 2};
  bool ok[2];
  T xn[2][3], xs[2][3], acc[2][3];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    ok[q] = i <= g.P.n[0] && j <= g.P.n[1] && kq[q] <= g.P.n[2];
    if (!ok[q]) continue;
    xn[q][0] = __ldg(g.lt[0] + i);
    xn[q][1] = __ldg(g.lt[1] + j);
    xn[q][2] = __ldg(g.lt[2] + kq[q]);
    const int no[3] = {i, j, kq[q]};
    T u[3];
    sample_velocity_node<T, TV>(g, V, no, T(S.ct[0]), u);  // first stage on the node
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (NOFF == 0) {
        xs[q][c] = xn[q][c] + dt * u[c];
      } else if (NOFF == 1) {
        xs[q][c] = xn[q][c] + HALF * dt * u[c];
      } else {
        const T k = dt * u[c];
        acc[q][c] = xn[q][c] + SIXTH * k;
        xs[q][c] = xn[q][c] + HALF * k;
      }
    }
  }
  unsigned parity = 0;
  bool alive = true;
#pragma unroll
  for (int s = 1; s <= NOFF; s++) {
    // (no break: the loop must unroll, so that V.cs[s] indexes the kernel parameters by constants)
    if (alive) alive = __syncthreads_and(mbar_wait_bounded(&bar, parity));
    if (!alive) continue;
    parity ^= 1u;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      if (!ok[q]) continue;
      const int no[3] = {i, j, kq[q]};
      T u[3];
      SplineStencil<T> st;
      if (!spline_stencil<T, 4, UNI>(g, sa, xs[q], no, st)) {
        u[0] = u[1] = u[2] = T(0);
      } else if (slt_inside(b, st.c0)) {
#pragma unroll
        for (int c = 0; c < 3; c++) u[c] = T(slt_apply<T, TV>(sa, st, tv + (size_t)c * slt_comp<TV>(), b, sx, sxy));
      } else {
#pragma unroll
        for (int c = 0; c < 3; c++) u[c] = T(spline_apply<T, 4, TV>(g, sa, st, V.cs[s][c]));
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const T k = dt * u[c];
        if (NOFF == 1) {  // RK2: x = xn + dt u(midpoint)
          xs[q][c] = xn[q][c] + dt * u[c];
        } else if (NOFF == 2) {  // RK3: stage 3 at xn + 2 k2 (src/lp_motion_m.f90:239-247)
          if (s == 1) {
            xs[q][c] = xn[q][c] + TWO * k;
            acc[q][c] = acc[q][c] + TWOTHIRD * k;
          } else {
            xs[q][c] = acc[q][c] + SIXTH * k;
          }
        } else {  // RK4
          if (s == 1) {
            acc[q][c] = acc[q][c] + THIRD * k;
            xs[q][c] = xn[q][c] + HALF * k;
          } else if (s == 2) {
            acc[q][c] = acc[q][c] + THIRD * k;
            xs[q][c] = xn[q][c] + k;
          } else {
            xs[q][c] = acc[q][c] + SIXTH * k;
          }
        }
      }
    }
    __syncthreads();  // every thread is done reading the box
    fence_proxy_async_smem();
    if (s < NOFF) slt_fill<TV>(tv, V.cs[s + 1][0], V.cs[s + 1][1], V.cs[s + 1][2], b, sx, sxy, &bar, tid);
    else slt_fill<T>(tf, fmo.f[0], fmo.f[1], fmo.f[2], b, sx, sxy, &bar, tid);
  }
  if (alive) {
    // departure points (xs now holds x): 2-D projection, particle BC, stick
#pragma unroll
    for (int q = 0; q < 2; q++) {
      if (!ok[q]) continue;
      int no[3] = {i, j, kq[q]};
      project_plane(g, no, xs[q]);
      if (particle_bc<T, HAS_FLAGS>(g, no, xs[q], err)) {
#pragma unroll
        for (int c = 0; c < 3; c++) xs[q][c] = xn[q][c];
      }
    }
    alive = __syncthreads_and(mbar_wait_bounded(&bar, parity));
  }
  if (!alive) {
    // a copy did not complete: record it, let the copies in flight land, and leave
    if (tid == 0) atomicOr(err, ERR_ASYNC_COPY);
    mbar_wait_bounded(&bar, parity);
    return;
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    if (!ok[q]) continue;
    const int k = kq[q];
    const int p = pidx(sx, sxy, i, j, k);
    const int nod[3] = {i, j, k};
    T fmp[3];
    SplineStencil<T> st;
    if (!spline_stencil<T, 4, UNI>(g, sa, xs[q], nod, st)) {
      fmp[0] = fmp[1] = fmp[2] = T(0);
    } else if (slt_inside(b, st.c0)) {
#pragma unroll
      for (int c = 0; c < 3; c++) fmp[c] = slt_apply<T, T>(sa, st, tf + (size_t)c * slt_comp<T>(), b, sx, sxy);
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) fmp[c] = spline_apply<T, 4>(g, sa, st, fmo.f[c]);
    }
    const int fl = HAS_FLAGS ? (int)g.flag[p] : (int)LCS_INTERNAL;
    const T mask = fl != LCS_MASK ? T(1) : T(0);
    const bool zero = HAS_FLAGS && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
    T vpre[3], vfin[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      vpre[c] = (fmp[c] + (xs[q][c] - xn[q][c])) * mask;
      vfin[c] = zero ? T(0) : vpre[c];
      fmn.f[c][p] = vfin[c];
    }
    write_ghosts<T, HAS_FLAGS, GHOST_FM>(g, fmn.f, i, j, k, vpre, vfin, err);
  }
}

}  // namespace cfd2lcs
