// Host set-up of a B-spline interpolation axis (knots, band LU, reciprocal spans).
#pragma once

#include <vector>

namespace cfd2lcs {

template <typename R>
struct SplineAxisHost {
  int n = 0, k = 0;
  std::vector<R> t;     // n + k knots
  std::vector<R> lu;    // (2k-1) x n band LU, column-major, diagonal in row k (1-based)
  std::vector<R> rinv;  // 6 reciprocal knot spans per interval
  std::vector<R> tu;    // per interval l, pair at 2(l-1): t(l), and 1/h where the knots the basis
                        // depends on are equally spaced by h (else 0)
  // x: strictly increasing abscissae (the padded coordinate line); order k.
  bool build(const std::vector<R> &x, int order);
};

}  // namespace cfd2lcs
