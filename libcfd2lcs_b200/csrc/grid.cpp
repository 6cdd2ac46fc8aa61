// Host-side grid setup: tensor-product restatement of init_sgrid (src/sgrid_m.f90:16-444)
// and compute_delta_xyz (:951-1014) for one rank.  See grid.h.
#include "grid.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace cfd2lcs {

namespace {

// Direction class of a padded index along an axis: -1 below, 0 interior, +1 above.
inline int side_of(int v, int n) { return v < 1 ? -1 : (v > n ? 1 : 0); }

}  // namespace

template <typename R>
R HostGrid<R>::coord(int c, int i, int j, int k) const {
  const int idx[3] = {i, j, k};
  const int v = idx[c];
  if (v >= 1 && v <= P.n[c]) return lt[c][v];
  if (c == P.single_axis) {
    // extrusion by (v-1) * unit(v1 x v2) * scaling, src/sgrid_m.f90:312-359; v1 and v2 are
    // central differences of the grid along the two in-plane directions at this cell's
    // in-plane indices (read on the lines through node 1), so the sign can change where a
    // periodic ghost coordinate is not translated
    auto diff = [&](int a, int w) {
      const int lo = std::max(w - 1, 0), hi = std::min(w + 1, P.n[a] + 1);
      return lt[a][hi] - lt[a][lo];
    };
    R cr;
    if (c == 0) cr = diff(1, j) * diff(2, k);
    else if (c == 1) cr = -(diff(0, i) * diff(2, k));
    else cr = diff(0, i) * diff(1, j);
    const R unit = cr > R(0) ? R(1) : (cr < R(0) ? R(-1) : R(0));
    return lt[c][1] + (R(v - 1) * unit) * scaling;
  }
  int e = 1;
  for (int a = 0; a < 3; a++)
    if (side_of(idx[a], P.n[a]) != 0 && !P.per[a]) e = 0;
  return P.gx[c][v < 1 ? 0 : 1][e];
}

template <typename R>
bool HostGrid<R>::build(const int n[3], const R *x, const R *y, const R *z, const int *fl) {
  error.clear();
  for (int a = 0; a < 3; a++) {
    if (n[a] < 1) {
      error = "init: ng > ni, nj or nk";
      return false;
    }
    P.n[a] = n[a];
  }
  P.sx = n[0] + 2;
  P.sxy = (n[0] + 2) * (n[1] + 2);
  const long npad = (long)(n[0] + 2) * (n[1] + 2) * (n[2] + 2);
  if (npad >= (1L << 31)) {
    error = "init: grid too large for 32-bit padded indexing";
    return false;
  }
  const long N = (long)n[0] * n[1] * n[2];
  auto at = [&](int i, int j, int k) { return (long)(i - 1) + (long)n[0] * ((j - 1) + (long)n[1] * (k - 1)); };

  int nsingle = 0;
  P.single_axis = -1;
  for (int a = 0; a < 3; a++)
    if (n[a] == 1) {
      nsingle++;
      P.single_axis = a;
    }
  if (nsingle > 1) {
    error = "init: more than one singleton direction (1-D grids) is not supported";
    return false;
  }

  // --- coordinate lines and the tensor-product test --------------------------------------
  // The reference accepts "rectilinear" grids within a 1e-4 tolerance
  // (check_rectilinear, src/sgrid_m.f90:868-949); the device path stores coordinate lines
  // and needs an exact tensor product.
  std::vector<R> line[3];
  for (int a = 0; a < 3; a++) line[a].assign(n[a] + 2, R(0));
  for (int i = 1; i <= n[0]; i++) line[0][i] = x[at(i, 1, 1)];
  for (int j = 1; j <= n[1]; j++) line[1][j] = y[at(1, j, 1)];
  for (int k = 1; k <= n[2]; k++) line[2][k] = z[at(1, 1, k)];
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++) {
        const long s = at(i, j, k);
        if (x[s] != line[0][i] || y[s] != line[1][j] || z[s] != line[2][k]) {
          error = "init: grid is not an exact tensor product of coordinate lines (curvilinear grids need "
                  "least-squares gradients, which this library does not provide)";
          return false;
        }
      }
  for (int a = 0; a < 3; a++)
    for (int i = 1; i < n[a]; i++)
      if (!(line[a][i + 1] > line[a][i])) {
        error = "init: coordinate lines must be strictly increasing";
        return false;
      }
  rectilinear = true;

  // --- periodicity from flags, src/sgrid_m.f90:107-136 ------------------------------------
  bool pl[6] = {false, false, false, false, false, false};
  bool any_flag = false;
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++) {
        const int f = fl[at(i, j, k)];
        if (f < LCS_INTERNAL || f > LCS_MASK) {
          error = "init: unknown bcflag value";
          return false;
        }
        if (f != LCS_INTERNAL) {
          any_flag = true;
          continue;
        }
        if (i == 1) pl[0] = true;
        if (j == 1) pl[1] = true;
        if (k == 1) pl[2] = true;
        if (i == n[0]) pl[3] = true;
        if (j == n[1]) pl[4] = true;
        if (k == n[2]) pl[5] = true;
      }
  for (int a = 0; a < 3; a++)
    if (pl[a] != pl[a + 3]) {
      error = "init: periodicity does not appear to match; check flag values passed to cfd2lcs_init";
      return false;
    }
  for (int a = 0; a < 3; a++) P.per[a] = (pl[a] && n[a] != 1) ? 1 : 0;
  P.zquirk = (P.per[2] && !P.per[1]) ? 1 : 0;

  // --- ghost coordinates ---------------------------------------------------------------
  // mirror ("fake") value, src/sgrid_m.f90:182-214: x(b) + (x(b) - x(ib)), ib the point
  // reflected through the boundary point b.
  R mir[3][2], img[3][2];
  for (int a = 0; a < 3; a++) {
    const int m = n[a];
    const R *L = line[a].data();
    mir[a][0] = L[1] + (L[1] - L[std::min(2, m)]);
    mir[a][1] = L[m] + (L[m] - L[std::max(m - 1, 1)]);
    img[a][0] = L[m];  // ghost 0 receives the slab at index n
    img[a][1] = L[1];  // ghost n+1 receives the slab at index 1
  }
  // periodic shifts from the first (untranslated) exchange, src/sgrid_m.f90:257-293:
  // shift of the ghost on side s of axis a = image - mirror
  R shift[3][2];
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) shift[a][s] = P.per[a] ? img[a][s] - mir[a][s] : R(0);
  for (int dk = -1; dk <= 1; dk++)
    for (int dj = -1; dj <= 1; dj++)
      for (int di = -1; di <= 1; di++) {
        const int d[3] = {di, dj, dk};
        bool ex = true;
        for (int a = 0; a < 3; a++)
          if (d[a] != 0 && !P.per[a]) ex = false;
        R *ps = P.ps[(dk + 1) * 9 + (dj + 1) * 3 + (di + 1)];
        for (int a = 0; a < 3; a++) ps[a] = (ex && d[a] != 0) ? shift[a][d[a] < 0 ? 0 : 1] : R(0);
      }
  // second exchange adds the shift of the packing direction (the opposite side); the z
  // component is read at direction (i,k,k) (src/comms_m.f90:750), which is zero unless y is
  // periodic too.
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      P.gx[a][s][0] = mir[a][s];
      R tr = img[a][s] + shift[a][1 - s];
      if (a == 2 && P.zquirk) tr = img[a][s];
      P.gx[a][s][1] = P.per[a] ? tr : mir[a][s];
    }
  // extrusion of the singleton direction, src/sgrid_m.f90:304-359
  if (P.single_axis >= 0) {
    R span = R(0);
    for (int a = 0; a < 3; a++) span = std::max(span, R(line[a][n[a]] - line[a][1]));
    scaling = span / R(std::max(std::max(n[0], n[1]), n[2]));
    const int a = P.single_axis;
    // unit normal v1 x v2 of the two in-plane directions: +x for a singleton x, -y for a
    // singleton y (x cross z), +z for a singleton z (x cross y), on increasing lines
    const R sign = (a == 1) ? R(-1) : R(1);
    for (int e = 0; e < 2; e++) {
      P.gx[a][0][e] = P.gx[a][0][e] + (R(-1) * sign) * scaling;
      P.gx[a][1][e] = P.gx[a][1][e] + (R(1) * sign) * scaling;
    }
  }
  for (int a = 0; a < 3; a++) {
    lt[a] = line[a];
    lt[a][0] = P.gx[a][0][P.per[a]];
    lt[a][n[a] + 1] = P.gx[a][1][P.per[a]];
    li[a] = lt[a];
    if (n[a] == 1) {  // fake unit spacing of interp_s2u_r1, src/lp_tracking_m.f90:367-378
      li[a][0] = li[a][1] - R(1.0);
      li[a][2] = li[a][1] + R(1.0);
    }
  }

  // --- bounding box over every padded node, src/sgrid_m.f90:362-372 ----------------------
  // Interior coordinates are the lines; ghost values are visited on the padded shell.
  for (int a = 0; a < 3; a++) {
    P.bb[a] = std::numeric_limits<R>::max();
    P.bb[a + 3] = -std::numeric_limits<R>::max();
    for (int v = 1; v <= n[a]; v++) {
      P.bb[a] = std::min(P.bb[a], lt[a][v]);
      P.bb[a + 3] = std::max(P.bb[a + 3], lt[a][v]);
    }
  }
  for (int k = 0; k <= n[2] + 1; k++)
    for (int j = 0; j <= n[1] + 1; j++) {
      const bool shell_jk = (k == 0 || k == n[2] + 1 || j == 0 || j == n[1] + 1);
      for (int i = 0; i <= n[0] + 1; i++) {
        if (!shell_jk && i != 0 && i != n[0] + 1) {
          i = n[0];  // skip the interior of this row (i jumps to n+1 next)
          continue;
        }
        for (int a = 0; a < 3; a++) {
          const R v = coord(a, i, j, k);
          P.bb[a] = std::min(P.bb[a], v);
          P.bb[a + 3] = std::max(P.bb[a + 3], v);
        }
      }
    }

  // --- inverse half spans for the CFL, src/sgrid_m.f90:951-1014 --------------------------
  // invd[a][(v*4 + cb)*4 + cc]: index v along a, classes of the other two axes (bit 0: the
  // neighbourhood reaches index 0, bit 1: it reaches index n+1).
  auto cls = [&](int v, int m) { return (v - 1 == 0 ? 1 : 0) | (v + 1 == m + 1 ? 2 : 0); };
  for (int a = 0; a < 3; a++) {
    invd[a].assign((size_t)(n[a] + 2) * 16, R(0));
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    for (int v = 1; v <= n[a]; v++)
      for (int cb = 0; cb < 4; cb++)
        for (int cc = 0; cc < 4; cc++) {
          // representative indices of the classes along b and c
          auto rep = [&](int cl, int m) {
            if (cl == 3) return 1;  // m == 1: both neighbours are ghosts
            if (cl == 1) return 1;
            if (cl == 2) return m;
            return m >= 3 ? 2 : -1;  // interior class needs m >= 3
          };
          const int rb = rep(cb, n[b]), rc = rep(cc, n[c]);
          if (rb < 0 || rc < 0 || cls(rb, n[b]) != cb || cls(rc, n[c]) != cc) continue;
          R mx = -std::numeric_limits<R>::max(), mn = std::numeric_limits<R>::max();
          for (int dv = -1; dv <= 1; dv++)
            for (int db = -1; db <= 1; db++)
              for (int dc = -1; dc <= 1; dc++) {
                int idx[3];
                idx[a] = v + dv;
                idx[b] = rb + db;
                idx[c] = rc + dc;
                const R val = coord(a, idx[0], idx[1], idx[2]);
                mx = std::max(mx, val);
                mn = std::min(mn, val);
              }
          const R half = R(0.5) * std::fabs(mx - mn);
          invd[a][((size_t)v * 4 + cb) * 4 + cc] = half > R(0) ? R(1) / half : R(0);
        }
  }

  // --- padded bcflag, src/sgrid_m.f90:182-255 --------------------------------------------
  bool need_flags = any_flag || P.single_axis >= 0;
  P.has_flags = need_flags ? 1 : 0;
  P.maxtrack = 2 * std::max(std::max(n[0], n[1]), n[2]);
  flag.clear();
  bcnorm.clear();
  if (!need_flags) return true;
  flag.assign(npad, 0);
  for (int k = 0; k <= n[2] + 1; k++)
    for (int j = 0; j <= n[1] + 1; j++)
      for (int i = 0; i <= n[0] + 1; i++)
        flag[pidx(i, j, k)] = (int8_t)fl[at(clamp_index(i, n[0]), clamp_index(j, n[1]), clamp_index(k, n[2]))];
  if (P.single_axis >= 0) {
    const int a = P.single_axis;
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    for (int vc = 0; vc <= n[c] + 1; vc++)
      for (int vb = 0; vb <= n[b] + 1; vb++) {
        int idx[3];
        idx[b] = vb;
        idx[c] = vc;
        idx[a] = 1;
        const int f1 = flag[pidx(idx[0], idx[1], idx[2])];
        const int8_t v = (int8_t)(f1 == LCS_INTERNAL ? LCS_2D : f1);
        idx[a] = 0;
        flag[pidx(idx[0], idx[1], idx[2])] = v;
        idx[a] = 2;
        flag[pidx(idx[0], idx[1], idx[2])] = v;
      }
  }

  // --- boundary normals, src/sgrid_m.f90:385-419 (least-squares gradient of min(flag,1),
  // full connectivity, src/gradient_m.f90:114-217 and :297-335) ---------------------------
  bool need_norm = false;
  for (long p = 0; p < npad && !need_norm; p++)
    if (flag[p] == LCS_MASK || flag[p] == LCS_SLIP || flag[p] == LCS_WALL) need_norm = true;
  if (!need_norm) return true;
  bcnorm.assign((size_t)3 * npad, R(0));
  auto bc_at = [&](int i, int j, int k) -> R {
    // exchange_sdata(scomm_max_r0, bc): ghosts filled from the periodic image
    int e = 1, any = 0;
    const int idx[3] = {i, j, k};
    for (int a = 0; a < 3; a++)
      if (side_of(idx[a], n[a]) != 0) {
        any = 1;
        if (!P.per[a]) e = 0;
      }
    int ii = i, jj = j, kk = k;
    if (any && e) {
      ii = wrap_index(i, n[0]);
      jj = wrap_index(j, n[1]);
      kk = wrap_index(k, n[2]);
    }
    const int f = flag[pidx(ii, jj, kk)];
    return f == LCS_2D ? R(LCS_INTERNAL) : R(std::min(f, 1));
  };
  static const int NB[27][3] = {
      {0, 0, 0},   {-1, 0, 0},  {0, -1, 0}, {0, 0, -1}, {1, 0, 0},  {0, 1, 0},  {0, 0, 1},   {-1, -1, -1}, {0, -1, -1},
      {1, -1, -1}, {-1, 0, -1}, {1, 0, -1}, {-1, 1, -1}, {0, 1, -1}, {1, 1, -1}, {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},
      {1, 1, 0},   {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},  {-1, 0, 1}, {1, 0, 1},  {-1, 1, 1},  {0, 1, 1},   {1, 1, 1}};
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++) {
        const long p = pidx(i, j, k);
        const int f = flag[p];
        if (f != LCS_MASK && f != LCS_SLIP && f != LCS_WALL) continue;
        const R x0 = coord(0, i, j, k), y0 = coord(1, i, j, k), z0 = coord(2, i, j, k);
        R sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        for (int nb = 1; nb < 27; nb++) {
          const int ii = i + NB[nb][0], jj = j + NB[nb][1], kk = k + NB[nb][2];
          const R d0 = coord(0, ii, jj, kk) - x0, d1 = coord(1, ii, jj, kk) - y0, d2 = coord(2, ii, jj, kk) - z0;
          const R idw = R(1) / (d0 * d0 + d1 * d1 + d2 * d2);
          sxx = sxx + idw * d0 * d0;
          syy = syy + idw * d1 * d1;
          szz = szz + idw * d2 * d2;
          sxy = sxy + idw * d0 * d1;
          sxz = sxz + idw * d0 * d2;
          syz = syz + idw * d1 * d2;
        }
        const R sden = R(2) * sxy * sxz * syz + sxx * syy * szz - sxx * syz * syz - syy * sxz * sxz - szz * sxy * sxy;
        const R b0 = bc_at(i, j, k);
        R gx = 0, gy = 0, gz = 0;
        for (int nb = 1; nb < 27; nb++) {
          const int ii = i + NB[nb][0], jj = j + NB[nb][1], kk = k + NB[nb][2];
          const R d0 = coord(0, ii, jj, kk) - x0, d1 = coord(1, ii, jj, kk) - y0, d2 = coord(2, ii, jj, kk) - z0;
          const R idw = R(1) / (d0 * d0 + d1 * d1 + d2 * d2);
          const R wx = idw * ((syy * szz - syz * syz) * d0 + (sxz * syz - sxy * szz) * d1 + (sxy * syz - sxz * syy) * d2) / sden;
          const R wy = idw * ((sxz * syz - sxy * szz) * d0 + (sxx * szz - sxz * sxz) * d1 + (sxy * sxz - syz * sxx) * d2) / sden;
          const R wz = idw * ((sxy * syz - sxz * syy) * d0 + (sxy * sxz - syz * sxx) * d1 + (sxx * syy - sxy * sxy) * d2) / sden;
          const R df = bc_at(ii, jj, kk) - b0;
          gx = gx + df * wx;
          gy = gy + df * wy;
          gz = gz + df * wz;
        }
        const R mag = gx * gx + gy * gy + gz * gz;
        if (mag <= R(0)) {
          gx = gy = gz = R(0);
        } else {
          gx = gx / std::sqrt(mag);
          gy = gy / std::sqrt(mag);
          gz = gz / std::sqrt(mag);
        }
        bcnorm[p] = gx;
        bcnorm[npad + p] = gy;
        bcnorm[2 * npad + p] = gz;
      }
  (void)N;
  return true;
}

template struct HostGrid<double>;
template struct HostGrid<float>;

}  // namespace cfd2lcs
