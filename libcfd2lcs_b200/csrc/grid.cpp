// Host-side grid setup: init_sgrid (src/sgrid_m.f90:16-444) and compute_delta_xyz
// (:951-1014) for one rank, as coordinate lines for tensor-product grids and as full padded
// arrays for non-rectilinear ones.  See grid.h.
#include "grid.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace cfd2lcs {

namespace {

// Direction class of a padded index along an axis: -1 below, 0 interior, +1 above.
inline int side_of(int v, int n) { return v < 1 ? -1 : (v > n ? 1 : 0); }

// NBR_OFFSET (src/data_m.f90:124-152): the neighbour order of the least-squares sums
const int kNbr[27][3] = {
    {0, 0, 0},   {-1, 0, 0},  {0, -1, 0}, {0, 0, -1}, {1, 0, 0},  {0, 1, 0},  {0, 0, 1},   {-1, -1, -1}, {0, -1, -1},
    {1, -1, -1}, {-1, 0, -1}, {1, 0, -1}, {-1, 1, -1}, {0, 1, -1}, {1, 1, -1}, {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},
    {1, 1, 0},   {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},  {-1, 0, 1}, {1, 0, 1},  {-1, 1, 1},  {0, 1, 1},   {1, 1, 1}};

// Fortran NINT: half away from zero
template <typename R>
inline int nint(R v) {
  return (int)(v >= R(0) ? std::floor((double)v + 0.5) : -std::floor(-(double)v + 0.5));
}

}  // namespace

// compute_lsgw (src/gradient_m.f90:114-217) at interior node (i,j,k) over the neighbours
// first..last of NBR_OFFSET: inverse-distance weights 1/|dx|^2 and the closed-form solution of
// the 3x3 normal equations, w[nb][c] the weight of neighbour nb in derivative c.  Products and
// sums keep the reference's grouping (the squares of sum(dx**2) and idw*dx**2 first).
template <typename R>
void HostGrid<R>::lsq_weights(int i, int j, int k, int first, int last, R w[27][3]) const {
  const R x0 = coord(0, i, j, k), y0 = coord(1, i, j, k), z0 = coord(2, i, j, k);
  R sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
  for (int nb = first; nb <= last; nb++) {
    const int ii = i + kNbr[nb][0], jj = j + kNbr[nb][1], kk = k + kNbr[nb][2];
    const R d0 = coord(0, ii, jj, kk) - x0, d1 = coord(1, ii, jj, kk) - y0, d2 = coord(2, ii, jj, kk) - z0;
    const R idw = R(1) / (d0 * d0 + d1 * d1 + d2 * d2);
    sxx = sxx + idw * (d0 * d0);
    syy = syy + idw * (d1 * d1);
    szz = szz + idw * (d2 * d2);
    sxy = sxy + idw * d0 * d1;
    sxz = sxz + idw * d0 * d2;
    syz = syz + idw * d1 * d2;
  }
  const R sden = R(2) * sxy * sxz * syz + sxx * syy * szz - sxx * (syz * syz) - syy * (sxz * sxz) - szz * (sxy * sxy);
  for (int nb = first; nb <= last; nb++) {
    const int ii = i + kNbr[nb][0], jj = j + kNbr[nb][1], kk = k + kNbr[nb][2];
    const R d0 = coord(0, ii, jj, kk) - x0, d1 = coord(1, ii, jj, kk) - y0, d2 = coord(2, ii, jj, kk) - z0;
    const R idw = R(1) / (d0 * d0 + d1 * d1 + d2 * d2);
    w[nb][0] = idw * ((syy * szz - syz * syz) * d0 + (sxz * syz - sxy * szz) * d1 + (sxy * syz - sxz * syy) * d2) / sden;
    w[nb][1] = idw * ((sxz * syz - sxy * szz) * d0 + (sxx * szz - sxz * sxz) * d1 + (sxy * sxz - syz * sxx) * d2) / sden;
    w[nb][2] = idw * ((sxy * syz - sxz * syy) * d0 + (sxy * sxz - syz * sxx) * d1 + (sxx * syy - sxy * sxy) * d2) / sden;
  }
}

template <typename R>
R HostGrid<R>::coord(int c, int i, int j, int k) const {
  if (!X[c].empty()) return X[c][pidx(i, j, k)];
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
  // An exact tensor product takes the line form below; any other grid is built as full
  // padded arrays (build_curvilinear), which accepts it when check_rectilinear classes it as
  // non-rectilinear.
  std::vector<R> line[3];
  for (int a = 0; a < 3; a++) line[a].assign(n[a] + 2, R(0));
  for (int i = 1; i <= n[0]; i++) line[0][i] = x[at(i, 1, 1)];
  for (int j = 1; j <= n[1]; j++) line[1][j] = y[at(1, j, 1)];
  for (int k = 1; k <= n[2]; k++) line[2][k] = z[at(1, 1, k)];
  bool tensor = true;
  for (int k = 1; k <= n[2] && tensor; k++)
    for (int j = 1; j <= n[1] && tensor; j++)
      for (int i = 1; i <= n[0]; i++) {
        const long s = at(i, j, k);
        if (x[s] != line[0][i] || y[s] != line[1][j] || z[s] != line[2][k]) {
          tensor = false;
          break;
        }
      }
  for (int a = 0; a < 3 && tensor; a++)
    for (int i = 1; i < n[a]; i++)
      if (!(line[a][i + 1] > line[a][i])) {
        error = "init: coordinate lines must be strictly increasing";
        return false;
      }
  rectilinear = tensor;
  P.curv = tensor ? 0 : 1;
  for (int c = 0; c < 3; c++) {
    X[c].clear();
    invdp[c].clear();
    pnorm[c].clear();
  }
  lsw.clear();

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
  if (!tensor) {
    if (!build_curvilinear(x, y, z)) return false;
  } else {
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
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++) {
        const long p = pidx(i, j, k);
        const int f = flag[p];
        if (f != LCS_MASK && f != LCS_SLIP && f != LCS_WALL) continue;
        R w[27][3];
        lsq_weights(i, j, k, 1, 26, w);
        const R b0 = bc_at(i, j, k);
        R gx = 0, gy = 0, gz = 0;
        for (int nb = 1; nb < 27; nb++) {
          const R df = bc_at(i + kNbr[nb][0], j + kNbr[nb][1], k + kNbr[nb][2]) - b0;
          gx = gx + df * w[nb][0];
          gy = gy + df * w[nb][1];
          gz = gz + df * w[nb][2];
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

// The non-rectilinear grid: init_sgrid's ghost construction on full padded arrays
// (src/sgrid_m.f90:169-372), check_rectilinear (:868-949), compute_delta_xyz (:951-1014), the
// face-neighbour least-squares weights (compute_lsgw with full_conn = .false., :421-424), the
// plane normals of project_lp2plane (src/lp_m.f90:446-486) and the node-guess constants of
// exchange_lp_alltoall (src/comms_m.f90:1625-1673).  P.n, P.per and the strides are set.
template <typename R>
bool HostGrid<R>::build_curvilinear(const R *x, const R *y, const R *z) {
  const int *n = P.n;
  const long npad = ntot();
  auto at = [&](int i, int j, int k) { return (long)(i - 1) + (long)n[0] * ((j - 1) + (long)n[1] * (k - 1)); };
  auto inside = [&](int i, int j, int k) { return i >= 1 && j >= 1 && k >= 1 && i <= n[0] && j <= n[1] && k <= n[2]; };
  auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
  const R *src[3] = {x, y, z};
  for (int c = 0; c < 3; c++) X[c].assign(npad, R(0));
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++)
        for (int c = 0; c < 3; c++) X[c][pidx(i, j, k)] = src[c][at(i, j, k)];
  // mirrored ghosts: x(b) + (x(b) - x(ib)), b the clamped node and ib its reflection
  for (int k = 0; k <= n[2] + 1; k++)
    for (int j = 0; j <= n[1] + 1; j++)
      for (int i = 0; i <= n[0] + 1; i++) {
        if (inside(i, j, k)) continue;
        const int ib = clampi(i, 1, n[0]), jb = clampi(j, 1, n[1]), kb = clampi(k, 1, n[2]);
        const long pb = pidx(ib, jb, kb);
        const long pr = pidx(clampi(2 * ib - i, 1, n[0]), clampi(2 * jb - j, 1, n[1]), clampi(2 * kb - k, 1, n[2]));
        for (int c = 0; c < 3; c++) X[c][pidx(i, j, k)] = X[c][pb] + (X[c][pb] - X[c][pr]);
      }
  // periodic images, exchange_sdata with max connectivity: per direction d whose non-zero
  // components are all periodic, the interior slab next to face d lands on the ghost slab
  // opposite, plus (second pass) the shift of d with its z component read at (i,k,k)
  auto dir = [](int di, int dj, int dk) { return (dk + 1) * 9 + (dj + 1) * 3 + (di + 1); };
  auto exchange = [&](bool translate) {
    for (int ic = 1; ic < 27; ic++) {
      const int d[3] = {kNbr[ic][0], kNbr[ic][1], kNbr[ic][2]};
      bool self = true;
      for (int a = 0; a < 3; a++)
        if (d[a] != 0 && !P.per[a]) self = false;
      if (!self) continue;
      int lo[3], hi[3];
      for (int a = 0; a < 3; a++) {
        lo[a] = d[a] == 1 ? n[a] : 1;
        hi[a] = d[a] == -1 ? 1 : n[a];
      }
      R sh[3] = {R(0), R(0), R(0)};
      if (translate) {
        sh[0] = P.ps[dir(d[0], d[1], d[2])][0];
        sh[1] = P.ps[dir(d[0], d[1], d[2])][1];
        sh[2] = P.ps[dir(d[0], d[2], d[2])][2];
      }
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            const long s0 = pidx(i, j, k), s1 = pidx(i - d[0] * n[0], j - d[1] * n[1], k - d[2] * n[2]);
            for (int c = 0; c < 3; c++) X[c][s1] = X[c][s0] + sh[c];
          }
    }
  };
  std::vector<R> mirror[3] = {X[0], X[1], X[2]};
  for (int q = 0; q < 27; q++)
    for (int c = 0; c < 3; c++) P.ps[q][c] = R(0);
  exchange(false);
  for (int kk = -1; kk <= 1; kk++)
    for (int jj = -1; jj <= 1; jj++)
      for (int ii = -1; ii <= 1; ii++) {
        const int gi = ii < 0 ? 0 : (ii == 0 ? 1 : n[0] + 1);
        const int gj = jj < 0 ? 0 : (jj == 0 ? 1 : n[1] + 1);
        const int gk = kk < 0 ? 0 : (kk == 0 ? 1 : n[2] + 1);
        const long p = pidx(gi, gj, gk);
        for (int c = 0; c < 3; c++) P.ps[dir(ii, jj, kk)][c] = X[c][p] - mirror[c][p];
      }
  exchange(true);
  // extrusion of a singleton direction by (v-1) * unit(v1 x v2) * scaling, v1 and v2 the
  // central differences along the in-plane directions on the lines through node 1
  {
    R span = R(0);
    for (int c = 0; c < 3; c++) {
      R mx = -std::numeric_limits<R>::max(), mn = std::numeric_limits<R>::max();
      for (int k = 1; k <= n[2]; k++)
        for (int j = 1; j <= n[1]; j++)
          for (int i = 1; i <= n[0]; i++) {
            mx = std::max(mx, X[c][pidx(i, j, k)]);
            mn = std::min(mn, X[c][pidx(i, j, k)]);
          }
      span = std::max(span, mx - mn);
    }
    scaling = span / R(std::max(std::max(n[0], n[1]), n[2]));
    auto cross_unit = [](const R v1[3], const R v2[3], R out[3]) {
      out[0] = v1[1] * v2[2] - v1[2] * v2[1];
      out[1] = v1[2] * v2[0] - v1[0] * v2[2];
      out[2] = v1[0] * v2[1] - v1[1] * v2[0];
      const R m = std::sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
      if (m > R(0))
        for (int c = 0; c < 3; c++) out[c] = out[c] / m;
    };
    for (int k = 0; k <= n[2] + 1; k++)
      for (int j = 0; j <= n[1] + 1; j++)
        for (int i = 0; i <= n[0] + 1; i++) {
          const int im = std::max(i - 1, 0), ip = std::min(i + 1, n[0] + 1);
          const int jm = std::max(j - 1, 0), jp = std::min(j + 1, n[1] + 1);
          const int km = std::max(k - 1, 0), kp = std::min(k + 1, n[2] + 1);
          R dl[3] = {R(0), R(0), R(0)}, v1[3], v2[3], cu[3];
          auto diff = [&](int i1, int j1, int k1, int i0, int j0, int k0, R out[3]) {
            for (int c = 0; c < 3; c++) out[c] = X[c][pidx(i1, j1, k1)] - X[c][pidx(i0, j0, k0)];
          };
          if (n[0] == 1 && i != 1) {
            diff(1, jp, 1, 1, jm, 1, v1);
            diff(1, 1, kp, 1, 1, km, v2);
            cross_unit(v1, v2, cu);
            for (int c = 0; c < 3; c++) dl[c] = R(i - 1) * cu[c];
          }
          if (n[1] == 1 && j != 1) {
            diff(ip, 1, 1, im, 1, 1, v1);
            diff(1, 1, kp, 1, 1, km, v2);
            cross_unit(v1, v2, cu);
            for (int c = 0; c < 3; c++) dl[c] = R(j - 1) * cu[c];
          }
          if (n[2] == 1 && k != 1) {
            diff(ip, 1, 1, im, 1, 1, v1);
            diff(1, jp, 1, 1, jm, 1, v2);
            cross_unit(v1, v2, cu);
            for (int c = 0; c < 3; c++) dl[c] = R(k - 1) * cu[c];
          }
          const long p = pidx(i, j, k);
          for (int c = 0; c < 3; c++) X[c][p] = X[c][p] + dl[c] * scaling;
        }
  }
  // bounding box over every padded node
  for (int c = 0; c < 3; c++) {
    P.bb[c] = std::numeric_limits<R>::max();
    P.bb[c + 3] = -std::numeric_limits<R>::max();
    for (long p = 0; p < npad; p++) {
      P.bb[c] = std::min(P.bb[c], X[c][p]);
      P.bb[c + 3] = std::max(P.bb[c + 3], X[c][p]);
    }
  }
  // check_rectilinear with its 1e-4 tolerance; the z lines run over 1..nk+1 (the loop index
  // the reference's z test reuses after its y loop)
  {
    R big = R(0);
    for (int c = 0; c < 3; c++) big = std::max(big, P.bb[c + 3] - P.bb[c]);
    const R tol = R(1e-4f);  // TOL = 1e-4, a default-real (single precision) literal
    bool ortho[3] = {true, true, true};
    const int lim[3] = {n[0], n[1], n[2] + 1};
    for (int a = 0; a < 3; a++) {
      const int b = a == 0 ? 1 : 0, c2 = a == 2 ? 1 : 2;  // the other two directions, b < c2
      for (int v2 = 1; v2 <= n[c2] && ortho[a]; v2++)
        for (int v1 = 1; v1 <= n[b] && ortho[a]; v1++) {
          R mx[3] = {-std::numeric_limits<R>::max(), -std::numeric_limits<R>::max(), -std::numeric_limits<R>::max()};
          R mn[3] = {std::numeric_limits<R>::max(), std::numeric_limits<R>::max(), std::numeric_limits<R>::max()};
          for (int v = 1; v <= lim[a]; v++) {
            int idx[3];
            idx[a] = v;
            idx[b] = v1;
            idx[c2] = v2;
            for (int c = 0; c < 3; c++) {
              const R val = X[c][pidx(idx[0], idx[1], idx[2])];
              mx[c] = std::max(mx[c], val);
              mn[c] = std::min(mn[c], val);
            }
          }
          for (int c = 0; c < 3; c++)
            if (c != a && std::fabs(mx[c] - mn[c]) / big > tol) ortho[a] = false;
        }
    }
    if (ortho[0] && ortho[1] && ortho[2]) {
      error = "init: the grid is rectilinear within check_rectilinear's 1e-4 tolerance but not an exact tensor product of "
              "coordinate lines; rectilinear grids need exact coordinate lines here";
      return false;
    }
  }
  // inverse half spans per node
  for (int c = 0; c < 3; c++) {
    invdp[c].assign(npad, R(0));
    for (int k = 1; k <= n[2]; k++)
      for (int j = 1; j <= n[1]; j++)
        for (int i = 1; i <= n[0]; i++) {
          R mx = -std::numeric_limits<R>::max(), mn = std::numeric_limits<R>::max();
          for (int kk = k - 1; kk <= k + 1; kk++)
            for (int jj = j - 1; jj <= j + 1; jj++)
              for (int ii = i - 1; ii <= i + 1; ii++) {
                mx = std::max(mx, X[c][pidx(ii, jj, kk)]);
                mn = std::min(mn, X[c][pidx(ii, jj, kk)]);
              }
          const R half = R(0.5) * std::fabs(mx - mn);
          invdp[c][pidx(i, j, k)] = half > R(0) ? R(1) / half : R(0);
        }
  }
  // face-neighbour least-squares weights
  lsw.assign((size_t)18 * npad, R(0));
  for (int k = 1; k <= n[2]; k++)
    for (int j = 1; j <= n[1]; j++)
      for (int i = 1; i <= n[0]; i++) {
        R w[27][3];
        lsq_weights(i, j, k, 1, 6, w);
        for (int nb = 1; nb <= 6; nb++)
          for (int c = 0; c < 3; c++) lsw[(size_t)((nb - 1) * 3 + c) * npad + pidx(i, j, k)] = w[nb][c];
      }
  // unit normal of the data plane of a 2-D grid at each interior node, v1 x v2 / |v1 x v2|
  // with v1, v2 the central differences along the two in-plane directions
  if (P.single_axis >= 0) {
    const int sa = P.single_axis;
    const int a1 = sa == 0 ? 1 : 0, a2 = sa == 2 ? 1 : 2;
    for (int c = 0; c < 3; c++) pnorm[c].assign(npad, R(0));
    for (int k = 1; k <= n[2]; k++)
      for (int j = 1; j <= n[1]; j++)
        for (int i = 1; i <= n[0]; i++) {
          int p1[3] = {i, j, k}, m1[3] = {i, j, k}, p2[3] = {i, j, k}, m2[3] = {i, j, k};
          p1[a1]++;
          m1[a1]--;
          p2[a2]++;
          m2[a2]--;
          R v1[3], v2[3];
          for (int c = 0; c < 3; c++) {
            v1[c] = X[c][pidx(p1[0], p1[1], p1[2])] - X[c][pidx(m1[0], m1[1], m1[2])];
            v2[c] = X[c][pidx(p2[0], p2[1], p2[2])] - X[c][pidx(m2[0], m2[1], m2[2])];
          }
          const R nx = v1[1] * v2[2] - v1[2] * v2[1], ny = v1[2] * v2[0] - v1[0] * v2[2], nz = v1[0] * v2[1] - v1[1] * v2[0];
          const R mag = std::sqrt(nx * nx + ny * ny + nz * nz);
          const long p = pidx(i, j, k);
          pnorm[0][p] = nx / mag;
          pnorm[1][p] = ny / mag;
          pnorm[2][p] = nz / mag;
        }
  }
  // exchange_lp_alltoall's node guess: index positions (from 1, ghosts included) of the first
  // smallest and largest value of each coordinate
  {
    R imin[3][3], imax[3][3];  // [coordinate][direction]
    for (int c = 0; c < 3; c++) {
      long pmin = 0, pmax = 0;
      for (long p = 1; p < npad; p++) {
        if (X[c][p] < X[c][pmin]) pmin = p;
        if (X[c][p] > X[c][pmax]) pmax = p;
      }
      const long pp[2] = {pmin, pmax};
      for (int e = 0; e < 2; e++) {
        const long p = pp[e];
        const R pos[3] = {R(p % P.sx + 1), R((p / P.sx) % (n[1] + 2) + 1), R(p / P.sxy + 1)};
        for (int a = 0; a < 3; a++) (e == 0 ? imin : imax)[c][a] = pos[a];
      }
    }
    const R third = R(1) / R(3);
    for (int a = 0; a < 3; a++) {
      P.guess0[a] = nint(third * (imin[0][a] + imin[1][a] + imin[2][a]));
      for (int c = 0; c < 3; c++) P.guessd[a][c] = imax[c][a] - imin[c][a];
    }
  }
  // coordinate lines through node 1, zero span tables and ghost constants: the line-based
  // kernels do not run on this grid, and these keep any table a launch receives in bounds
  for (int a = 0; a < 3; a++) {
    lt[a].assign(n[a] + 2, R(0));
    for (int v = 0; v <= n[a] + 1; v++) {
      int idx[3] = {1, 1, 1};
      idx[a] = v;
      lt[a][v] = X[a][pidx(idx[0], idx[1], idx[2])];
    }
    li[a] = lt[a];
    invd[a].assign((size_t)(n[a] + 2) * 16, R(0));
    for (int s2 = 0; s2 < 2; s2++)
      for (int e = 0; e < 2; e++) P.gx[a][s2][e] = lt[a][s2 == 0 ? 0 : n[a] + 1];
  }
  return true;
}

template struct HostGrid<double>;
template struct HostGrid<float>;

}  // namespace cfd2lcs
