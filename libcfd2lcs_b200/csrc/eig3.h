// Largest eigenvalue of a real symmetric 3x3 matrix in closed form, for the FTLE
// (compute_ftle, src/lcs_m.f90:160-177, where the reference calls LAPACK DSYEV per point and
// keeps W(3)).  Method: the trigonometric solution of the characteristic cubic
// (O. K. Smith, "Eigenvalues of a symmetric 3 x 3 matrix", Comm. ACM 4(4):168, 1961): with
// q = tr(A)/3, B = A - qI and p = sqrt(tr(B^2)/6), the eigenvalues are q + 2p cos(phi + 2k pi/3)
// with phi = acos(r)/3, r = det(B/p)/2, the largest at k = 0.  The matrix is first scaled by a
// power of two (exact) so that its largest entry lies in [0.5, 1): no intermediate over- or
// underflows for any finite input.  A NaN entry gives NaN.
// Where the two largest eigenvalues (nearly) coincide, r -> -1 and acos amplifies the rounding
// of r to about sqrt(eps) in the result; there (r < -1 + 1e-3, where the amplification would
// exceed 0.41/sqrt(1+r) ~ 13 units of rounding of p) the value comes from a cyclic Jacobi
// iteration instead, whose accuracy does not depend on the spacing of the eigenvalues.
// Accuracy: a few units of rounding relative to the largest |eigenvalue| (the FTLE's
// Cauchy-Green tensor is positive semi-definite, so that is a relative bound on the value
// used); tests/test_eig3.py checks both paths against LAPACK on random, near-degenerate and
// wide-range matrices.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define CFD2LCS_HD __host__ __device__
#else
#define CFD2LCS_HD
#endif

namespace cfd2lcs {

// Cyclic Jacobi on the symmetric 3x3 (rotations zeroing (0,1), (0,2), (1,2) in turn) until
// the off-diagonal part is below 1e-18 of the diagonal, at most 32 sweeps; the largest
// diagonal entry.
CFD2LCS_HD inline double eig3_max_jacobi(double a00, double a01, double a02, double a11, double a12, double a22) {
  using std::fabs;
  using std::sqrt;
  double a[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
  for (int sweep = 0; sweep < 32; sweep++) {
    const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
    if (off == 0.0 || off <= 1e-18 * diag) break;
    for (int pq = 0; pq < 3; pq++) {
      const int pp = pq == 2 ? 1 : 0, qq = pq == 0 ? 1 : 2;
      const double apq = a[pp][qq];
      if (apq == 0.0) continue;
      const double theta = (a[qq][qq] - a[pp][pp]) / (2.0 * apq);
      const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      for (int r = 0; r < 3; r++) {
        const double arp = a[r][pp], arq = a[r][qq];
        a[r][pp] = c * arp - s * arq;
        a[r][qq] = s * arp + c * arq;
      }
      for (int r = 0; r < 3; r++) {
        const double apr = a[pp][r], aqr = a[qq][r];
        a[pp][r] = c * apr - s * aqr;
        a[qq][r] = s * apr + c * aqr;
      }
    }
  }
  return fmax(fmax(a[0][0], a[1][1]), a[2][2]);
}

CFD2LCS_HD inline double eig3_max_closed(double a00, double a01, double a02, double a11, double a12, double a22) {
  using std::acos;
  using std::cos;
  using std::fabs;
  using std::sqrt;
  const double m = fmax(fmax(fmax(fabs(a00), fabs(a01)), fmax(fabs(a02), fabs(a11))), fmax(fabs(a12), fabs(a22)));
  if (!(m > 0.0)) return m == 0.0 ? 0.0 : a00 + a01 + a02 + a11 + a12 + a22;  // zero matrix, or NaN
  if (m > 1.0e300) return a00 + a01 + a02 + a11 + a12 + a22 - m + m;       // infinite entries
  int e = 0;
  (void)std::frexp(m, &e);
  const double s = std::ldexp(1.0, -e), inv = std::ldexp(1.0, e);
  a00 *= s;
  a01 *= s;
  a02 *= s;
  a11 *= s;
  a12 *= s;
  a22 *= s;
  const double q = (a00 + a11 + a22) / 3.0;
  const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
  const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
  const double p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1;
  if (!(p2 > 0.0)) return q * inv;  // A = qI
  const double p = sqrt(p2 / 6.0);
  const double det = b00 * (b11 * b22 - a12 * a12) - a01 * (a01 * b22 - a12 * a02) + a02 * (a01 * a12 - b11 * a02);
  double r = det / (2.0 * p * p * p);
  if (r < -1.0 + 1e-3) return eig3_max_jacobi(a00, a01, a02, a11, a12, a22) * inv;  // two largest (nearly) equal
  r = fmin(r, 1.0);
  return (q + 2.0 * p * cos(acos(r) / 3.0)) * inv;
}

}  // namespace cfd2lcs
