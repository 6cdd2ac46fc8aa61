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

#include <cuda.h>  // CUtensorMap (the descriptor type only; maps are encoded by the engine)

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

// one 3-D box of a tensor map (coordinates x, y, z in elements; out-of-range parts read as 0)
// to 128-byte aligned shared dst
__device__ __forceinline__ void tensor_copy_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// orders this thread's earlier shared-memory accesses before later bulk copies into them
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---------------------------------------------------------------------------------------
// Staged boxes: a block of TX x TY x TZ nodes copies the box of its nodes widened by HALO on
// every side, one row (x line) per bulk copy.  A row copy starts at the 16-byte boundary at or
// below its first element, so a row in shared memory is preceded by up to 16/sizeof - 1
// extra elements (its alignment shift, (xlo + y sx + z sxy) mod 16/sizeof).
// ---------------------------------------------------------------------------------------
template <int TX_, int TY_, int TZ_, int HALO_>
struct TileGeom {
  static constexpr int TX = TX_, TY = TY_, TZ = TZ_, HALO = HALO_;
  static constexpr int SX = TX + 2 * HALO, SY = TY + 2 * HALO, SZ = TZ + 2 * HALO;
  static constexpr int ROWS = SY * SZ;  // rows of the box per component
  template <typename TC>
  __host__ __device__ static constexpr int pitch() {
    return ((SX + 2 * (16 / (int)sizeof(TC) - 1)) / (16 / (int)sizeof(TC))) * (16 / (int)sizeof(TC));
  }
  template <typename TC>
  __host__ __device__ static constexpr int comp() {  // elements of one component
    return ROWS * pitch<TC>();
  }
};

// The staged box of a block: origin (padded indices, may lie outside the array) and the part
// inside the padded array, [lo, hi) per axis.
struct TileBox {
  int xs, ys, zs;
  int xlo, xhi, ylo, yhi, zlo, zhi;
};

template <typename G, typename T>
__device__ __forceinline__ TileBox tile_box(const DevGrid<T> &g) {
  TileBox b;
  b.xs = 1 + (int)blockIdx.x * G::TX - G::HALO;
  b.ys = 1 + (int)blockIdx.y * G::TY - G::HALO;
  b.zs = 1 + (int)blockIdx.z * G::TZ - G::HALO;
  b.xlo = max(b.xs, 0);
  b.xhi = min(b.xs + G::SX, g.P.sx);
  b.ylo = max(b.ys, 0);
  b.yhi = min(b.ys + G::SY, g.P.n[1] + 2);
  b.zlo = max(b.zs, 0);
  b.zhi = min(b.zs + G::SZ, g.P.n[2] + 2);
  return b;
}

// Issues the row copies of a 3-component field into buf (component c at buf + c * comp): the
// 3 * ROWS copies are dealt over the block's threads, each arriving once per copy on bar (with
// the row's bytes, or none for a row outside the padded array), so bar expects 3 * ROWS
// arrivals per field.
template <typename G, typename TC>
__device__ __forceinline__ void tile_fill(TC *buf, const TC *f0, const TC *f1, const TC *f2, const TileBox &b, int sx, int sxy,
                                          uint64_t *bar, int tid, int nthreads) {
  constexpr int E = 16 / (int)sizeof(TC);
  for (int task = tid; task < 3 * G::ROWS; task += nthreads) {
    const int c = task / G::ROWS, r = task - c * G::ROWS;
    const TC *const src = c == 0 ? f0 : (c == 1 ? f1 : f2);
    const int y = b.ys + r % G::SY, z = b.zs + r / G::SY;
    if (y >= b.ylo && y < b.yhi && z >= b.zlo && z < b.zhi && b.xhi > b.xlo) {
      const long e = (long)b.xlo + (long)y * sx + (long)z * sxy;
      const long a = e & ~(long)(E - 1);
      const unsigned bytes = (unsigned)((((e - a) + (b.xhi - b.xlo)) * (long)sizeof(TC) + 15) & ~15L);
      mbar_arrive_expect_tx(bar, bytes);
      bulk_copy_g2s(buf + (size_t)c * G::template comp<TC>() + (size_t)r * G::template pitch<TC>(), src + a, bytes, bar);
    } else {
      mbar_arrive(bar);
    }
  }
}

// Tensor maps of the staged fields of one launch (the engine encodes them; `on` = 0: copy the
// boxes row by row instead).  A map describes one padded component as a 3-D array with box
// (pitch, SY, SZ); it exists only where a row of the array is a multiple of 16 bytes, and then
// every row has the same alignment shift (xlo mod 16/sizeof), so a box copied from x0 = xlo
// rounded down to 16 bytes lands each element exactly where tile_index expects it.
struct TileMaps {
  CUtensorMap m[12];
  int on;
};

// The 3-component field of maps m[0..2] into buf: one box copy per component, all issued by
// thread 0, which arrives once on bar with their bytes.
template <typename G, typename TC>
__device__ __forceinline__ void tile_fill_tensor(TC *buf, const CUtensorMap *m, const TileBox &b, uint64_t *bar, int tid) {
  if (tid != 0) return;
  constexpr int E = 16 / (int)sizeof(TC);
  constexpr unsigned bytes = (unsigned)(G::ROWS * G::template pitch<TC>() * sizeof(TC));
  mbar_arrive_expect_tx(bar, 3 * bytes);
  const int x0 = b.xlo & ~(E - 1);
#pragma unroll
  for (int c = 0; c < 3; c++) tensor_copy_3d(buf + (size_t)c * G::template comp<TC>(), m + c, x0, b.ys, b.zs, bar);
}

// 128-byte aligned start of the dynamic shared memory (box copies need it); launches ask for
// 128 bytes more than their boxes
__device__ __forceinline__ unsigned char *smem_aligned128(unsigned char *p) {
  return reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(p) + 127) & ~(uintptr_t)127);
}

// shared-memory index of padded element (x, y, z) of a staged component
template <typename G, typename TC>
__device__ __forceinline__ int tile_index(const TileBox &b, int sx, int sxy, int x, int y, int z) {
  constexpr int E = 16 / (int)sizeof(TC);
  return ((z - b.zs) * G::SY + (y - b.ys)) * G::template pitch<TC>() + ((b.xlo + y * sx + z * sxy) & (E - 1)) + (x - b.xlo);
}

// ---------------------------------------------------------------------------------------
// Cubic tile geometry: 32 x 4 x 4 nodes (block of 32 x 4 x 2 threads, 2 nodes each), halo 2
// ---------------------------------------------------------------------------------------
using CubicGeom = TileGeom<32, 4, 4, 2>;
constexpr int SLT_X = CubicGeom::TX, SLT_Y = CubicGeom::TY, SLT_Z = CubicGeom::TZ;
constexpr int SLT_THREADS = 256;
template <typename TC>
__host__ __device__ constexpr int slt_pitch() {
  return CubicGeom::pitch<TC>();
}
template <typename TC>
__host__ __device__ constexpr int slt_comp() {
  return CubicGeom::comp<TC>();
}
// shared memory of one staged field (3 components); the flow map's type is the widest
template <typename TC>
__host__ __device__ constexpr size_t slt_field_bytes() {
  return (size_t)3 * slt_comp<TC>() * sizeof(TC);
}

// true when the stencil's 4 x 4 x 4 coefficients are all in the staged box
__device__ __forceinline__ bool slt_inside(const TileBox &b, const int c0[3]) {
  return c0[0] >= b.xlo && c0[0] + 4 <= b.xhi && c0[1] >= b.ylo && c0[1] + 4 <= b.yhi && c0[2] >= b.zlo && c0[2] + 4 <= b.zhi;
}

// One component from the staged box of geometry G: coefficient (x, y, z) sits in row
// (z-zs)*SY + (y-ys) at column x - xlo plus the row's alignment shift
// ((xlo + y sx + z sxy) mod 16/sizeof).
template <typename G, typename T, typename TC>
__device__ __forceinline__ TC tile_apply(const SplineAxes<T> &sa, const SplineStencil<T> &st, const TC *comp, const TileBox &b, int sx,
                                         int sxy) {
  constexpr int E = 16 / (int)sizeof(TC);
  const int gy = st.c0[1] * sx + st.c0[2] * sxy + b.xlo;  // global offset of row (c0y, c0z) at column xlo
  const int rb = ((st.c0[2] - b.zs) * G::SY + (st.c0[1] - b.ys)) * G::template pitch<TC>() + (st.c0[0] - b.xlo);
  return spline_contract<T, 4, TC>(sa, st, [&](int c1, int c2, int c0) {
    const int shift = (gy + c1 * sx + c2 * sxy) & (E - 1);
    return comp[rb + (c2 * G::SY + c1) * G::template pitch<TC>() + shift + c0];
  });
}

template <typename T, typename TC>
__device__ __forceinline__ TC slt_apply(const SplineAxes<T> &sa, const SplineStencil<T> &st, const TC *comp, const TileBox &b, int sx,
                                        int sxy) {
  return tile_apply<CubicGeom, T, TC>(sa, st, comp, b, sx, sxy);
}

// Two vertical neighbours whose stencils share the x and y intervals and sit one z row apart
// (B.c0 = A.c0 + (0, 0, 1), the common case: neighbouring nodes move alike): one pass over the
// 5 z rows they span reads each shared tap once (80 shared-memory loads instead of 2 x 64)
// and accumulates both points in spline_contract's order (c2, c1, c0 increasing), so each
// result has the bits of its own contraction.
template <typename T, typename TC>
__device__ __forceinline__ void slt_apply_pair(const SplineStencil<T> &A, const SplineStencil<T> &B, const TC *comp, const TileBox &b,
                                               int sx, int sxy, TC &oa, TC &ob) {
  constexpr int E = 16 / (int)sizeof(TC);
  const int gy = A.c0[1] * sx + A.c0[2] * sxy + b.xlo;
  const int rb = ((A.c0[2] - b.zs) * CubicGeom::SY + (A.c0[1] - b.ys)) * slt_pitch<TC>() + (A.c0[0] - b.xlo);
  TC vza = TC(0), vzb = TC(0);
#pragma unroll
  for (int c2 = 0; c2 < 5; c2++) {
    TC vya = TC(0), vyb = TC(0);
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) {
      const int shift = (gy + c1 * sx + c2 * sxy) & (E - 1);
      const TC *row = comp + rb + (c2 * CubicGeom::SY + c1) * slt_pitch<TC>() + shift;
      TC vxa = TC(0), vxb = TC(0);
#pragma unroll
      for (int c0 = 0; c0 < 4; c0++) {
        const TC tap = row[c0];
        if (c2 < 4) vxa += TC(A.b[0][c0]) * tap;
        if (c2 > 0) vxb += TC(B.b[0][c0]) * tap;
      }
      if (c2 < 4) vya += TC(A.b[1][c1]) * vxa;
      if (c2 > 0) vyb += TC(B.b[1][c1]) * vxb;
    }
    if (c2 < 4) vza += TC(A.b[2][c2]) * vya;
    if (c2 > 0) vzb += TC(B.b[2][c2 - 1]) * vyb;
  }
  oa = vza;
  ob = vzb;
}

// A 3-component field (staged box `box`, global arrays g0..g2) at the thread's two points
// x[q] around nodes (i, j, kq[q]): the pair pass where it applies, else each point from the box
// or, when its stencil leaves the box, from global memory; 0 where db3val returns 0.
template <typename T, typename TC, bool UNI>
__device__ __forceinline__ void slt_sample2(const DevGrid<T> &g, const SplineAxes<T> &sa, const TileBox &b, const TC *box, const TC *g0,
                                            const TC *g1, const TC *g2, const bool ok[2], const T x[2][3], int i, int j,
                                            const int kq[2], T out[2][3]) {
  const int sx = g.P.sx, sxy = g.P.sxy;
  SplineStencil<T> st[2];
  bool in[2], inbox[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int no[3] = {i, j, kq[q]};
    in[q] = ok[q] && spline_stencil<T, 4, UNI>(g, sa, x[q], no, st[q]);
    inbox[q] = in[q] && slt_inside(b, st[q].c0);
    if (!in[q]) out[q][0] = out[q][1] = out[q][2] = T(0);
  }
  if (inbox[0] && inbox[1] && st[0].c0[0] == st[1].c0[0] && st[0].c0[1] == st[1].c0[1] && st[1].c0[2] == st[0].c0[2] + 1) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      TC a, bb;
      slt_apply_pair<T, TC>(st[0], st[1], box + (size_t)c * slt_comp<TC>(), b, sx, sxy, a, bb);
      out[0][c] = T(a);
      out[1][c] = T(bb);
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    if (!in[q]) continue;
    if (inbox[q]) {
#pragma unroll
      for (int c = 0; c < 3; c++) out[q][c] = T(slt_apply<T, TC>(sa, st[q], box + (size_t)c * slt_comp<TC>(), b, sx, sxy));
    } else {
      out[q][0] = T(spline_apply<T, 4, TC>(g, sa, st[q], g0));
      out[q][1] = T(spline_apply<T, 4, TC>(g, sa, st[q], g1));
      out[q][2] = T(spline_apply<T, 4, TC>(g, sa, st[q], g2));
    }
  }
}

#ifndef CFD2LCS_SLT_MINB
#define CFD2LCS_SLT_MINB 2
#endif

template <typename T, typename TV, int INTEG, bool HAS_FLAGS>
__global__ void __launch_bounds__(SLT_THREADS, CFD2LCS_SLT_MINB)
    k_sl_tile(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, FieldPtrs<T> fmo, FieldPtrsW<T> fmn, StageTimes S, T dt, int *err,
              const __grid_constant__ TileMaps tm) {
  extern __shared__ __align__(128) unsigned char slt_smem_raw[];
  unsigned char *const slt_smem = smem_aligned128(slt_smem_raw);
  __shared__ __align__(8) uint64_t bar;
  constexpr bool UNI = uniform_basis<T, TV>();
  constexpr int NOFF = INTEG == RK2_ ? 1 : (INTEG == RK3_ ? 2 : (INTEG == RK4_ ? 3 : 0));  // stages off the node
  const T HALF = T(1) / T(2), THIRD = T(1) / T(3), TWOTHIRD = T(2) / T(3), SIXTH = T(1) / T(6), TWO = T(2);
  const int tid = threadIdx.x + 32 * (threadIdx.y + SLT_Y * threadIdx.z);
  const int sx = g.P.sx, sxy = g.P.sxy;
  const TileBox b = tile_box<CubicGeom>(g);
  const int I0 = 1 + (int)blockIdx.x * SLT_X, J0 = 1 + (int)blockIdx.y * SLT_Y, K0 = 1 + (int)blockIdx.z * SLT_Z;
  TV *const tv = reinterpret_cast<TV *>(slt_smem);
  T *const tf = reinterpret_cast<T *>(slt_smem);
  if (tid == 0) mbar_init(&bar, tm.on ? 1 : 3 * CubicGeom::ROWS);
  __syncthreads();
  // field f: the blend of off-node stage f + 1 (f < NOFF), then the flow map (f = NOFF); maps 3f..3f+2
  auto fill = [&](int f) {
    if (tm.on) {
      if (f < NOFF) tile_fill_tensor<CubicGeom, TV>(tv, tm.m + 3 * f, b, &bar, tid);
      else tile_fill_tensor<CubicGeom, T>(tf, tm.m + 3 * f, b, &bar, tid);
    } else if (f < NOFF) {
      tile_fill<CubicGeom, TV>(tv, V.cs[f + 1][0], V.cs[f + 1][1], V.cs[f + 1][2], b, sx, sxy, &bar, tid, SLT_THREADS);
    } else {
      tile_fill<CubicGeom, T>(tf, fmo.f[0], fmo.f[1], fmo.f[2], b, sx, sxy, &bar, tid, SLT_THREADS);
    }
  };
  fill(0);

  // the thread's two nodes: vertical neighbours (i, j, k) and (i, j, k + 1)
  const int i = I0 + (int)threadIdx.x, j = J0 + (int)threadIdx.y;
  const int kq[2] = {K0 + 2 * (int)threadIdx.z, K0 + 2 * (int)threadIdx.z + 1};
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
    T us[2][3];
    slt_sample2<T, TV, UNI>(g, sa, b, tv, V.cs[s][0], V.cs[s][1], V.cs[s][2], ok, xs, i, j, kq, us);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      if (!ok[q]) continue;
      const T *u = us[q];
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
    fill(s);
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
  T fms[2][3];
  slt_sample2<T, T, UNI>(g, sa, b, tf, fmo.f[0], fmo.f[1], fmo.f[2], ok, xs, i, j, kq, fms);
#pragma unroll
  for (int q = 0; q < 2; q++) {
    if (!ok[q]) continue;
    const int k = kq[q];
    const int p = pidx(sx, sxy, i, j, k);
    const T *fmp = fms[q];
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

// ---------------------------------------------------------------------------------------
// LINEAR backward subcycle from a staged box (interp_s2u_r1 LINEAR, src/lp_tracking_m.f90:
// 342-474, inside update_flowmap_sl): the bracket of every stage and of the departure point
// is [no-1, no] or [no, no+1] around the node (clamped t), so a block of 32 x 4 x 4 nodes reads
// only the box of its nodes widened by 1 -- for both velocity levels and the previous flow map.
// The block copies the nine component boxes with one mbarrier phase, then every point runs
// from shared memory with the expressions of k_sl_subcycle (lin_blend_contract, lin_contract),
// so the results are bitwise equal.  The gathering kernel is latency-bound (three dependent
// gather phases per point); here the only global reads are the bulk copies.
// ---------------------------------------------------------------------------------------
// One node (i, j, k) of the LINEAR backward subcycle from staged taps: integrate_lp
// (src/lp_motion_m.f90:129-360) with the stage placement of integrate<>, the first stage on the
// node (sample_velocity_node), the trilinear samples of interp_s2u_r1 LINEAR
// (src/lp_tracking_m.f90:342-474) around the node from its interpolation lines lm, lc, lp at
// no-1, no, no+1, then the previous flow map at the departure point, the boundary rules and the
// ghost writes.  rm / rp are the reciprocal spans of the lines' brackets below and above the
// node (DevGrid::ri at no-1 and no).  iv / ifm map a padded (x, y, z) to the staged index of a velocity / flow-map
// component; u0 / u1 / fm (c, index) read component c of u_n, u_np1 and the flow map.  Every
// staged LINEAR kernel runs this one expression, so they are bitwise equal to each other and to
// k_sl_subcycle.
template <typename T, typename TV, int INTEG, bool HAS_FLAGS, typename IV, typename IF, typename U0, typename U1, typename FM>
__device__ __forceinline__ void lin_sl_node(const DevGrid<T> &g, const StageTimes &S, T dt, int i, int j, int k, const T xn[3], const T lm[3],
                                            const T lc[3], const T lp[3], const T rm[3], const T rp[3], IV iv, IF ifm, U0 u0, U1 u1, FM fm,
                                            FieldPtrsW<T> fmn, int *err) {
  constexpr int NOFF = INTEG == RK2_ ? 1 : (INTEG == RK3_ ? 2 : (INTEG == RK4_ ? 3 : 0));
  const T HALF = T(1) / T(2), THIRD = T(1) / T(3), TWOTHIRD = T(2) / T(3), SIXTH = T(1) / T(6), TWO = T(2);
  const int sx = g.P.sx, sxy = g.P.sxy;
  const int no[3] = {i, j, k};
  auto vel_sample = [&](const T x[3], T ct_, T u[3]) {
    const TV ct = TV(ct_), omc = TV(1) - ct;
    LinStencil<T> st;
    lin_stencil_node(lm, lc, lp, rm, rp, sx, sxy, x, no, st);
    int idx[8];
#pragma unroll
    for (int c = 0; c < 8; c++)
      idx[c] = iv(st.i0[0] + ((c & 1) ? st.d[0] : 0), st.i0[1] + ((c & 2) ? st.d[1] : 0), st.i0[2] + ((c & 4) ? st.d[2] : 0));
#pragma unroll
    for (int c = 0; c < 3; c++)
      u[c] = T(lin_blend_contract<T, TV>(st, omc, ct, [&](int e) { return u0(c, idx[e]); }, [&](int e) { return u1(c, idx[e]); }));
  };
  T u[3], x[3];
  {  // first stage on the node (sample_velocity_node)
    const TV ct = TV(T(S.ct[0])), omc = TV(1) - ct;
    const int pv = iv(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; c++) u[c] = T(omc * u0(c, pv) + ct * u1(c, pv));
  }
  if (NOFF == 0) {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = xn[c] + dt * u[c];
  } else if (NOFF == 1) {
    T xh[3];
#pragma unroll
    for (int c = 0; c < 3; c++) xh[c] = xn[c] + HALF * dt * u[c];
    vel_sample(xh, T(S.ct[1]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = xn[c] + dt * u[c];
  } else if (NOFF == 2) {
    T kk[3], xs[3], acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      acc[c] = xn[c] + SIXTH * kk[c];
      xs[c] = xn[c] + HALF * kk[c];
    }
    vel_sample(xs, T(S.ct[1]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      xs[c] = xn[c] + TWO * kk[c];
      acc[c] = acc[c] + TWOTHIRD * kk[c];
    }
    vel_sample(xs, T(S.ct[2]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * kk[c];
    }
  } else {
    T kk[3], xs[3], acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      acc[c] = xn[c] + SIXTH * kk[c];
      xs[c] = xn[c] + HALF * kk[c];
    }
    vel_sample(xs, T(S.ct[1]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      acc[c] = acc[c] + THIRD * kk[c];
      xs[c] = xn[c] + HALF * kk[c];
    }
    vel_sample(xs, T(S.ct[2]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      acc[c] = acc[c] + THIRD * kk[c];
      xs[c] = xn[c] + kk[c];
    }
    vel_sample(xs, T(S.ct[3]), u);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      kk[c] = dt * u[c];
      x[c] = acc[c] + SIXTH * kk[c];
    }
  }
  int nb[3] = {i, j, k};
  project_plane(g, nb, x);
  if (particle_bc<T, HAS_FLAGS>(g, nb, x, err)) {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = xn[c];
  }
  // previous flow map at the departure point (sample_field LINEAR around the node)
  LinStencil<T> st;
  lin_stencil_node(lm, lc, lp, rm, rp, sx, sxy, x, no, st);
  int idx[8];
#pragma unroll
  for (int c = 0; c < 8; c++)
    idx[c] = ifm(st.i0[0] + ((c & 1) ? st.d[0] : 0), st.i0[1] + ((c & 2) ? st.d[1] : 0), st.i0[2] + ((c & 4) ? st.d[2] : 0));
  T fmp[3];
#pragma unroll
  for (int c = 0; c < 3; c++) fmp[c] = lin_contract<T>(st, [&](int e) { return fm(c, idx[e]); });
  const int p = pidx(sx, sxy, i, j, k);
  const int fl = HAS_FLAGS ? (int)g.flag[p] : (int)LCS_INTERNAL;
  const T mask = fl != LCS_MASK ? T(1) : T(0);
  const bool zero = HAS_FLAGS && (fl == LCS_MASK || fl == LCS_INFLOW || fl == LCS_OUTFLOW);
  T vpre[3], vfin[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    vpre[c] = (fmp[c] + (x[c] - xn[c])) * mask;
    vfin[c] = zero ? T(0) : vpre[c];
    fmn.f[c][p] = vfin[c];
  }
  write_ghosts<T, HAS_FLAGS, GHOST_FM>(g, fmn.f, i, j, k, vpre, vfin, err);
}

using LinGeom = TileGeom<32, 4, 4, 1>;

// shared memory of the LINEAR tile: u_n, u_np1 (velocity type) and the flow map (3 each)
template <typename T, typename TV>
__host__ __device__ constexpr size_t sll_bytes() {
  return (size_t)6 * LinGeom::comp<TV>() * sizeof(TV) + (size_t)3 * LinGeom::comp<T>() * sizeof(T);
}

#ifndef CFD2LCS_SLL_MINB
#define CFD2LCS_SLL_MINB 2
#endif

template <typename T, typename TV, int INTEG, bool HAS_FLAGS>
__global__ void __launch_bounds__(SLT_THREADS, CFD2LCS_SLL_MINB)
    k_sl_tile_lin(DevGrid<T> g, VelFields<TV> V, FieldPtrs<T> fmo, FieldPtrsW<T> fmn, StageTimes S, T dt, int *err,
                  const __grid_constant__ TileMaps tm) {
  extern __shared__ __align__(128) unsigned char sll_smem_raw[];
  unsigned char *const sll_smem = smem_aligned128(sll_smem_raw);
  __shared__ __align__(8) uint64_t bar;
  const int tid = threadIdx.x + 32 * (threadIdx.y + LinGeom::TY * threadIdx.z);
  const int sx = g.P.sx, sxy = g.P.sxy;
  const TileBox b = tile_box<LinGeom>(g);
  TV *const su0 = reinterpret_cast<TV *>(sll_smem);
  TV *const su1 = su0 + 3 * LinGeom::comp<TV>();
  T *const sf = reinterpret_cast<T *>(sll_smem + (size_t)6 * LinGeom::comp<TV>() * sizeof(TV));
  if (tid == 0) mbar_init(&bar, tm.on ? 3 : 9 * LinGeom::ROWS);
  __syncthreads();
  if (tm.on) {  // maps 0-2: u_n, 3-5: u_np1, 6-8: flow map
    tile_fill_tensor<LinGeom, TV>(su0, tm.m, b, &bar, tid);
    tile_fill_tensor<LinGeom, TV>(su1, tm.m + 3, b, &bar, tid);
    tile_fill_tensor<LinGeom, T>(sf, tm.m + 6, b, &bar, tid);
  } else {
    tile_fill<LinGeom, TV>(su0, V.un[0], V.un[1], V.un[2], b, sx, sxy, &bar, tid, SLT_THREADS);
    tile_fill<LinGeom, TV>(su1, V.unp1[0], V.unp1[1], V.unp1[2], b, sx, sxy, &bar, tid, SLT_THREADS);
    tile_fill<LinGeom, T>(sf, fmo.f[0], fmo.f[1], fmo.f[2], b, sx, sxy, &bar, tid, SLT_THREADS);
  }

  const int I0 = 1 + (int)blockIdx.x * LinGeom::TX, J0 = 1 + (int)blockIdx.y * LinGeom::TY, K0 = 1 + (int)blockIdx.z * LinGeom::TZ;
  const int i = I0 + (int)threadIdx.x, j = J0 + (int)threadIdx.y;
  const int kq[2] = {K0 + (int)threadIdx.z, K0 + (int)threadIdx.z + 2};
  bool ok[2];
  T xn[2][3];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    ok[q] = i <= g.P.n[0] && j <= g.P.n[1] && kq[q] <= g.P.n[2];
    xn[q][0] = __ldg(g.lt[0] + min(i, g.P.n[0] + 1));
    xn[q][1] = __ldg(g.lt[1] + min(j, g.P.n[1] + 1));
    xn[q][2] = __ldg(g.lt[2] + min(kq[q], g.P.n[2] + 1));
  }
  if (!__syncthreads_and(mbar_wait_bounded(&bar, 0))) {
    if (tid == 0) atomicOr(err, ERR_ASYNC_COPY);
    mbar_wait_bounded(&bar, 0);  // let the copies in flight land before the block leaves
    return;
  }
  // the interpolation lines at no-1, no, no+1 of both points (every bracket of a node's stages
  // and departure point lies there), read while the box copies are in flight
  T lm[2][3], lc[2][3], lp[2][3], rm[2][3], rp[2][3];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int nd[3] = {min(i, g.P.n[0]), min(j, g.P.n[1]), min(kq[q], g.P.n[2])};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      lm[q][a] = __ldg(g.li[a] + nd[a] - 1);
      lc[q][a] = __ldg(g.li[a] + nd[a]);
      lp[q][a] = __ldg(g.li[a] + nd[a] + 1);
      rm[q][a] = __ldg(g.ri[a] + nd[a] - 1);
      rp[q][a] = __ldg(g.ri[a] + nd[a]);
    }
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    if (!ok[q]) continue;
    lin_sl_node<T, TV, INTEG, HAS_FLAGS>(
        g, S, dt, i, j, kq[q], xn[q], lm[q], lc[q], lp[q], rm[q], rp[q],
        [&](int x, int y, int z) { return tile_index<LinGeom, TV>(b, sx, sxy, x, y, z); },
        [&](int x, int y, int z) { return tile_index<LinGeom, T>(b, sx, sxy, x, y, z); },
        [&](int c, int e) { return su0[(size_t)c * LinGeom::comp<TV>() + e]; },
        [&](int c, int e) { return su1[(size_t)c * LinGeom::comp<TV>() + e]; },
        [&](int c, int e) { return sf[(size_t)c * LinGeom::comp<T>() + e]; }, fmn, err);
  }
}

// ---------------------------------------------------------------------------------------
// LINEAR backward subcycle marching along z (FP64 with tensor maps).  A block owns a column of
// 32 x 8 nodes over a run of kc planes and keeps a ring of four staged planes of all nine
// components (u_n, u_np1, flow map; each plane 34 x 10 with its 1-node halo): while it works on
// plane k from planes k-1, k and k+1, the copy of plane k+2 lands in the slot plane k-2 left.
// Against the 32 x 4 x 4 boxes of k_sl_tile_lin (34 x 6 x 6 staged per 512 nodes, 2.4 staged
// elements per node) a plane is staged once per column run, 1.33 elements per node in x and y,
// plus two planes per run in z, and the block never waits for its copies but at the start of a
// run.  Every copy lands on the mbarrier of its slot (one phase per plane that passes through
// it); every wait is bounded.
// ---------------------------------------------------------------------------------------
constexpr int SLM_X = 32, SLM_Y = 8, SLM_SX = SLM_X + 2, SLM_SY = SLM_Y + 2, SLM_SLOTS = 4;
constexpr int SLM_THREADS = SLM_X * SLM_Y;
// elements of one staged component plane, padded so that every copy lands 128-byte aligned
template <typename T>
__host__ __device__ constexpr int slm_comp() {
  return ((SLM_SX * SLM_SY * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T);
}
template <typename T>
__host__ __device__ constexpr size_t slm_bytes() {
  return (size_t)SLM_SLOTS * 9 * slm_comp<T>() * sizeof(T);
}

#ifndef CFD2LCS_SLM_MINB
#define CFD2LCS_SLM_MINB 2
#endif

template <typename T, int INTEG, bool HAS_FLAGS>
__global__ void __launch_bounds__(SLM_THREADS, CFD2LCS_SLM_MINB)
    k_sl_march_lin(DevGrid<T> g, FieldPtrsW<T> fmn, StageTimes S, T dt, int kc, int *err, const __grid_constant__ TileMaps tm) {
  extern __shared__ __align__(128) unsigned char slm_smem_raw[];
  T *const box = reinterpret_cast<T *>(smem_aligned128(slm_smem_raw));
  __shared__ __align__(8) uint64_t bar[SLM_SLOTS];
  constexpr int CS = slm_comp<T>();
  constexpr unsigned PLANE_BYTES = 9u * (unsigned)(SLM_SX * SLM_SY * sizeof(T));
  const int tid = threadIdx.x + SLM_X * threadIdx.y;
  const int xs = (int)blockIdx.x * SLM_X, ys = (int)blockIdx.y * SLM_Y;  // padded origin of the staged planes
  const int K0 = 1 + (int)blockIdx.z * kc, K1 = min(K0 + kc - 1, g.P.n[2]);
  // plane p (K0-1 <= p <= K1+1) sits in slot p & 3; its phase on that slot's barrier is the
  // parity of its pass through the ring
  auto parity = [&](int p) { return (unsigned)(((p - (K0 - 1)) >> 2) & 1); };
  auto issue = [&](int p) {
    T *const dst = box + (size_t)(p & 3) * 9 * CS;
    mbar_arrive_expect_tx(&bar[p & 3], PLANE_BYTES);
#pragma unroll
    for (int c = 0; c < 9; c++) tensor_copy_3d(dst + (size_t)c * CS, tm.m + c, xs, ys, p, &bar[p & 3]);
  };
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < SLM_SLOTS; s++) mbar_init(&bar[s], 1);
  }
  __syncthreads();
  if (tid == 0)
    for (int p = K0 - 1; p <= min(K0 + 1, K1 + 1); p++) issue(p);

  const int i = xs + 1 + (int)threadIdx.x, j = ys + 1 + (int)threadIdx.y;
  const bool ok = i <= g.P.n[0] && j <= g.P.n[1];
  // x and y stay fixed along the column: the node coordinates, the interpolation lines at
  // no-1, no, no+1 and the reciprocal spans of both axes are read once
  const int ni = min(i, g.P.n[0]), nj = min(j, g.P.n[1]);
  T xn[3], lm[3], lc[3], lp[3];
  xn[0] = __ldg(g.lt[0] + min(i, g.P.n[0] + 1));
  xn[1] = __ldg(g.lt[1] + min(j, g.P.n[1] + 1));
  lm[0] = __ldg(g.li[0] + ni - 1), lc[0] = __ldg(g.li[0] + ni), lp[0] = __ldg(g.li[0] + ni + 1);
  lm[1] = __ldg(g.li[1] + nj - 1), lc[1] = __ldg(g.li[1] + nj), lp[1] = __ldg(g.li[1] + nj + 1);
  T zc = __ldg(g.li[2] + K0 - 1), zp = __ldg(g.li[2] + K0);
  T rm[3], rp[3];
  rm[0] = __ldg(g.ri[0] + ni - 1), rp[0] = __ldg(g.ri[0] + ni);
  rm[1] = __ldg(g.ri[1] + nj - 1), rp[1] = __ldg(g.ri[1] + nj);
  T rz = __ldg(g.ri[2] + K0 - 1);
  auto sidx = [&](int x, int y, int z) { return (z & 3) * 9 * CS + (y - ys) * SLM_SX + (x - xs); };
  for (int k = K0; k <= K1; k++) {
    bool w = mbar_wait_bounded(&bar[(k + 1) & 3], parity(k + 1));
    if (k == K0) w = mbar_wait_bounded(&bar[(k - 1) & 3], parity(k - 1)) && mbar_wait_bounded(&bar[k & 3], parity(k)) && w;
    // the barrier also ends every thread's reads of plane k-2, whose slot the next copy fills
    if (!__syncthreads_and(w)) {
      if (tid == 0) atomicOr(err, ERR_ASYNC_COPY);
      // let the copies in flight land before the block leaves
      for (int p = max(K0 - 1, k - 1); p <= min(k + 1, K1 + 1); p++) mbar_wait_bounded(&bar[p & 3], parity(p));
      return;
    }
    if (tid == 0 && k + 2 <= K1 + 1) {
      fence_proxy_async_smem();
      issue(k + 2);
    }
    // z lines of this plane, rolled along the column
    lm[2] = zc;
    lc[2] = zp;
    zc = zp;
    zp = __ldg(g.li[2] + k + 1);
    lp[2] = zp;
    xn[2] = __ldg(g.lt[2] + k);
    rm[2] = rz;
    rz = __ldg(g.ri[2] + k);
    rp[2] = rz;
    if (ok)
      lin_sl_node<T, T, INTEG, HAS_FLAGS>(
          g, S, dt, i, j, k, xn, lm, lc, lp, rm, rp, sidx, sidx, [&](int c, int e) { return box[(size_t)c * CS + e]; },
          [&](int c, int e) { return box[(size_t)(3 + c) * CS + e]; }, [&](int c, int e) { return box[(size_t)(6 + c) * CS + e]; },
          fmn, err);
  }
}

// ---------------------------------------------------------------------------------------
// Forward particle subcycle with the B-spline taps staged in shared memory: the cubic form of
// k_fwd_subcycle (update_lp, src/lp_motion_m.f90:15-54, with integrate_lp and the CUBIC branch
// of interp_s2u_r1).  The particles are sorted by cell in tiles of 16 x 4 x 4 cells
// (k_particle_count / k_particle_scatter, every other subcycle); one block advances the
// particles of one tile.  At the sort a particle lies in its cell c; one unsorted subcycle and
// the RK stages move it at most 1.5 cells per axis (the CFL bound), so its stencils read the
// coefficients c-3 .. c+4: the tile widened by 4 cells (24 x 12 x 12 per component), which the
// block copies into shared memory once per RK stage -- the stage's blend -- with row bulk copies
// on an mbarrier.  Stencils outside the box read global memory; both paths run spline_contract,
// so the particles move bitwise as in k_fwd_subcycle.
// ---------------------------------------------------------------------------------------
using FwdGeom = TileGeom<16, 4, 4, 4>;
constexpr int FWT_TX = FwdGeom::TX, FWT_TY = FwdGeom::TY, FWT_TZ = FwdGeom::TZ;

template <typename TV>
__host__ __device__ constexpr size_t fwt_bytes() {
  return (size_t)3 * FwdGeom::comp<TV>() * sizeof(TV);
}

// the box of sort tile (tx, ty, tz): cells tx*TX .. widened by HALO - 1 below, HALO above
template <typename G, typename T>
__device__ __forceinline__ TileBox tile_box_at(const DevGrid<T> &g, int tx, int ty, int tz) {
  TileBox b;
  b.xs = 1 + tx * G::TX - G::HALO;
  b.ys = 1 + ty * G::TY - G::HALO;
  b.zs = 1 + tz * G::TZ - G::HALO;
  b.xlo = max(b.xs, 0);
  b.xhi = min(b.xs + G::SX, g.P.sx);
  b.ylo = max(b.ys, 0);
  b.yhi = min(b.ys + G::SY, g.P.n[1] + 2);
  b.zlo = max(b.zs, 0);
  b.zhi = min(b.zs + G::SZ, g.P.n[2] + 2);
  return b;
}

// one 3-component B-spline sample from a staged box (global memory where the stencil leaves it)
template <typename G, typename T, typename TC, bool UNI>
__device__ __forceinline__ void tile_sample1(const DevGrid<T> &g, const SplineAxes<T> &sa, const TileBox &b, const TC *box, const TC *g0,
                                             const TC *g1, const TC *g2, const T x[3], const int no[3], T out[3]) {
  SplineStencil<T> st;
  if (!spline_stencil<T, 4, UNI>(g, sa, x, no, st)) {
    out[0] = out[1] = out[2] = T(0);
    return;
  }
  if (slt_inside(b, st.c0)) {
#pragma unroll
    for (int c = 0; c < 3; c++) out[c] = T(tile_apply<G, T, TC>(sa, st, box + (size_t)c * G::template comp<TC>(), b, g.P.sx, g.P.sxy));
  } else {
    out[0] = T(spline_apply<T, 4, TC>(g, sa, st, g0));
    out[1] = T(spline_apply<T, 4, TC>(g, sa, st, g1));
    out[2] = T(spline_apply<T, 4, TC>(g, sa, st, g2));
  }
}

// One particle per thread in blocks of 512 (a tile holds about 256 particles, so a round rarely
// repeats), 2 resident blocks (64 registers) per SM: 32 warps, as the gathering kernel runs.
constexpr int FWT_THREADS = 512, FWT_PPT = 1;
#ifndef CFD2LCS_FWT_MINB
#define CFD2LCS_FWT_MINB 2
#endif

template <typename T, typename TV, int INTEG, bool HAS_FLAGS>
__global__ void __launch_bounds__(FWT_THREADS, CFD2LCS_FWT_MINB)
    k_fwd_tile(DevGrid<T> g, SplineAxes<T> sa, VelFields<TV> V, Particles<T> P, StageTimes S, T dt, const int *offs, const int *tsum,
               SortTiles st, int np, int *err, const __grid_constant__ TileMaps tm) {
  extern __shared__ __align__(128) unsigned char fwt_smem_raw[];
  unsigned char *const fwt_smem = smem_aligned128(fwt_smem_raw);
  __shared__ __align__(8) uint64_t bar;
  constexpr bool UNI = particle_uniform_basis();  // as k_fwd_subcycle
  constexpr int NS = INTEG == RK2_ ? 2 : (INTEG == RK3_ ? 3 : (INTEG == RK4_ ? 4 : 1));  // samples per step
  const T HALF = T(1) / T(2), THIRD = T(1) / T(3), TWOTHIRD = T(2) / T(3), SIXTH = T(1) / T(6), TWO = T(2);
  const long ntiles = (long)st.ntx * st.nty * st.ntz;
  const long t = blockIdx.x;
  const int start = sort_tile_start(offs, tsum, t, ntiles, np), end = sort_tile_start(offs, tsum, t + 1, ntiles, np);
  if (start >= end) return;  // an empty tile (the whole block leaves)
  const int tx = (int)(t % st.ntx), ty = (int)((t / st.ntx) % st.nty), tz = (int)(t / ((long)st.ntx * st.nty));
  const TileBox b = tile_box_at<FwdGeom>(g, tx, ty, tz);
  const int tid = threadIdx.x, sx = g.P.sx, sxy = g.P.sxy;
  TV *const tv = reinterpret_cast<TV *>(fwt_smem);
  if (tid == 0) mbar_init(&bar, tm.on ? 1 : 3 * FwdGeom::ROWS);
  __syncthreads();
  // the blend of stage s (maps 3s..3s+2)
  auto fill = [&](int s) {
    if (tm.on) tile_fill_tensor<FwdGeom, TV>(tv, tm.m + 3 * s, b, &bar, tid);
    else tile_fill<FwdGeom, TV>(tv, V.cs[s][0], V.cs[s][1], V.cs[s][2], b, sx, sxy, &bar, tid, FWT_THREADS);
  };
  unsigned parity = 0;
  bool alive = true;
  for (int r0 = start; r0 < end && alive; r0 += FWT_PPT * FWT_THREADS) {  // rounds (block-uniform)
    fill(0);
    int qs[FWT_PPT];
    bool ok[FWT_PPT];
    T xn[FWT_PPT][3], xs[FWT_PPT][3], acc[FWT_PPT][3];
    int no[FWT_PPT][3];
#pragma unroll
    for (int q = 0; q < FWT_PPT; q++) {
      qs[q] = r0 + q * FWT_THREADS + tid;
      ok[q] = qs[q] < end;
      if (!ok[q]) continue;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        xn[q][c] = P.x[c][qs[q]];
        xs[q][c] = xn[q][c];
        no[q][c] = P.no[c][qs[q]];
      }
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
      // (no break: the loop must unroll, so that V.cs[s] indexes the kernel parameters by constants)
      if (alive) alive = __syncthreads_and(mbar_wait_bounded(&bar, parity));
      if (!alive) continue;
      parity ^= 1u;
#pragma unroll
      for (int q = 0; q < FWT_PPT; q++) {
        if (!ok[q]) continue;
        T u[3];
        tile_sample1<FwdGeom, T, TV, UNI>(g, sa, b, tv, V.cs[s][0], V.cs[s][1], V.cs[s][2], xs[q], no[q], u);
        // integrate_lp (src/lp_motion_m.f90:129-360) with the stage placement of integrate<>
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const T k = dt * u[c];
          if (NS == 1) {
            xs[q][c] = xn[q][c] + dt * u[c];
          } else if (NS == 2) {
            xs[q][c] = s == 0 ? xn[q][c] + HALF * dt * u[c] : xn[q][c] + dt * u[c];
          } else if (NS == 3) {
            if (s == 0) {
              acc[q][c] = xn[q][c] + SIXTH * k;
              xs[q][c] = xn[q][c] + HALF * k;
            } else if (s == 1) {
              xs[q][c] = xn[q][c] + TWO * k;
              acc[q][c] = acc[q][c] + TWOTHIRD * k;
            } else {
              xs[q][c] = acc[q][c] + SIXTH * k;
            }
          } else {
            if (s == 0) {
              acc[q][c] = xn[q][c] + SIXTH * k;
              xs[q][c] = xn[q][c] + HALF * k;
            } else if (s == 1) {
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
      if (s + 1 < NS) fill(s + 1);
    }
    if (!alive) break;
    // project, particle BC, stick, displacement, one node-search pass, periodic wrap
#pragma unroll
    for (int q = 0; q < FWT_PPT; q++) {
      if (!ok[q]) continue;
      const int sl = qs[q];
      T *x = xs[q];
      int *nd = no[q];
      project_plane(g, nd, x);
      if (particle_bc<T, HAS_FLAGS>(g, nd, x, err)) {
#pragma unroll
        for (int c = 0; c < 3; c++) x[c] = xn[q][c];
      }
#pragma unroll
      for (int c = 0; c < 3; c++) P.dx[c][sl] = P.dx[c][sl] + (x[c] - xn[q][c]);
      track_pass(g, x, nd);
      wrap_particle(g, x, nd);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        P.x[c][sl] = x[c];
        P.no[c][sl] = nd[c];
      }
    }
  }
  if (!alive) {
    // a copy did not complete: record it, let the copies in flight land, and leave
    if (tid == 0) atomicOr(err, ERR_ASYNC_COPY);
    mbar_wait_bounded(&bar, parity);
  }
}

}  // namespace cfd2lcs
