// Host-side grid setup of libcfd2lcs_b200: the reference's init_sgrid (src/sgrid_m.f90:16-444)
// and compute_delta_xyz (:951-1014), one rank.
//
// A grid that is an exact tensor product of coordinate lines is stored as three lines plus
// the rules the reference's ghost construction produces: mirrored "fake" ghosts, periodic
// images with the periodic shift (including the z shift read at direction (i,k,k),
// src/comms_m.f90:750), and the extrusion of a singleton direction (src/sgrid_m.f90:304-359);
// those kernels never see full 3-D coordinate arrays.  Any other grid that the reference
// classes as non-rectilinear (check_rectilinear, :868-949) keeps the full padded coordinate
// arrays, built by the same ghost construction, together with what the reference's
// non-rectilinear path needs: face-neighbour least-squares gradient weights (compute_lsgw,
// src/gradient_m.f90:114-217), inverse half spans per node, the plane normals of a 2-D grid
// (project_lp2plane, src/lp_m.f90:418-538) and the node-guess constants of
// exchange_lp_alltoall (src/comms_m.f90:1625-1673).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cfd2lcs {

enum { LCS_INTERNAL = 0, LCS_INFLOW = 1, LCS_OUTFLOW = 2, LCS_WALL = 3, LCS_SLIP = 4, LCS_2D = 5, LCS_MASK = 6 };

// Small per-grid constants every kernel receives by value.
template <typename R>
struct GridParams {
  int n[3];           // interior points per direction
  int sx, sxy;        // padded strides: p = i + sx*j + sxy*k, i,j,k in [0, n+1]
  int per[3];         // periodic directions
  int single_axis;    // singleton direction (2-D grid) or -1
  int zquirk;         // z periodic but y not: periodic z ghosts carry no shift
  // Ghost coordinate of axis c on side s (0: index 0, 1: index n+1); e = 1 when the ghost
  // cell was filled by a periodic exchange (every out-of-range direction of the cell is
  // periodic), e = 0 when it kept its mirrored (and, for a singleton axis, extruded) value.
  R gx[3][2][2];
  R bb[6];            // bounding box of all coordinates including ghosts
  R ps[27][3];        // periodic shift per direction, index (dk+1)*9 + (dj+1)*3 + (di+1)
  int has_flags;      // bcflag array present (some flag is not LCS_INTERNAL or 2-D)
  int maxtrack;       // 2*max(n): recursion limit of the node search
  int curv;           // non-rectilinear grid: full coordinate arrays and least squares
  // non-rectilinear grids, exchange_lp_alltoall's node guess per direction a:
  // nint((imin_x + imin_y + imin_z)/3) and the index spans imax_c - imin_c of the coordinate
  // extremes (minloc / maxloc over the padded arrays, src/comms_m.f90:1625-1673)
  int guess0[3];
  R guessd[3][3];     // [direction a][coordinate c]
};

// RN(1 / (l[i+1] - l[i])) for i = 0 .. size-2 (0 where the span is 0, and at the last index):
// the reciprocal spans of an interpolation line, the table the LINEAR stencils' quotient
// (lin_quotient) reads.  R's own division, so the value is the correctly rounded reciprocal of
// the span the kernels form as l[i+1] - l[i].
template <typename R>
inline std::vector<R> reciprocal_spans(const std::vector<R> &l) {
  std::vector<R> r(l.size(), R(0));
  for (size_t i = 0; i + 1 < l.size(); i++) {
    const R b = l[i + 1] - l[i];
    r[i] = b != R(0) ? R(1) / b : R(0);
  }
  return r;
}

template <typename R>
struct HostGrid {
  GridParams<R> P{};
  // coordinate lines with ghosts (index 0 .. n+1):
  std::vector<R> lt[3];   // node coordinates for tracking, gradients and boundary conditions
  std::vector<R> li[3];   // interpolation lines (2-D: fake unit spacing, src/lp_tracking_m.f90:367-378)
  std::vector<R> invd[3]; // 1/half-span per index for x (by i) and y (by j)
  std::vector<R> invdz;   // 1/half-span for z, by (k, i class, j class): index (k*4 + ci)*4 + cj
  std::vector<int8_t> flag;  // padded bcflag (empty when has_flags == 0)
  std::vector<R> bcnorm;     // 3 x padded, only at nodes whose flag needs it (empty otherwise)
  // non-rectilinear grids only (empty otherwise), padded layout:
  std::vector<R> X[3];       // node coordinates (sgrid%grid)
  std::vector<R> lsw;        // 18 planes: weight of face neighbour nb (NBR_OFFSET 2..7) for
                             // derivative c at plane nb*3 + c, zero on the ghost layer
  std::vector<R> invdp[3];   // inverse half spans per node (compute_delta_xyz)
  std::vector<R> pnorm[3];   // 2-D grids: unit normal of the data plane at interior nodes
  bool rectilinear = false;
  R scaling = R(0);          // extrusion length of a singleton direction
  std::string error;         // non-empty: the grid is rejected

  // Builds everything from the caller's arrays (n[0]*n[1]*n[2] values, i fastest).
  bool build(const int n[3], const R *x, const R *y, const R *z, const int *flag_in);

  // Coordinate c of any node of the padded grid (the reference's sgrid%grid).
  R coord(int c, int i, int j, int k) const;

  // The non-rectilinear branch of build(): padded coordinates and their tables (above).
  bool build_curvilinear(const R *x, const R *y, const R *z);
  // Least-squares gradient weights at an interior node over NBR_OFFSET neighbours first..last.
  void lsq_weights(int i, int j, int k, int first, int last, R w[27][3]) const;
  long ntot() const { return (long)P.sxy * (P.n[2] + 2); }
  long pidx(int i, int j, int k) const { return (long)i + (long)P.sx * j + (long)P.sxy * k; }
};

// Rule of the reference's ghost fill for a padded field: exchange_sdata SELF copies for
// periodic directions, then set_velocity_bc / set_flowmap_bc by ghost flag.
inline int wrap_index(int g, int n) { return g < 1 ? g + n : (g > n ? g - n : g); }
inline int clamp_index(int g, int n) { return g < 1 ? 1 : (g > n ? n : g); }

}  // namespace cfd2lcs
