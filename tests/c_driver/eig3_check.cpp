// Host build of the library's closed-form 3x3 eigenvalue (libcfd2lcs_b200/csrc/eig3.h) for
// tests/test_eig3.py: reads lines of six numbers (a00 a01 a02 a11 a12 a22) from stdin and
// prints the largest eigenvalue of each with 17 significant digits, by the closed form (with its
// Jacobi fallback) and by the Jacobi iteration alone.
#include <cstdio>

#include "eig3.h"

int main() {
  double a[6];
  while (std::scanf("%lf %lf %lf %lf %lf %lf", a, a + 1, a + 2, a + 3, a + 4, a + 5) == 6)
    std::printf("%.17g %.17g\n", cfd2lcs::eig3_max_closed(a[0], a[1], a[2], a[3], a[4], a[5]),
                cfd2lcs::eig3_max_jacobi(a[0], a[1], a[2], a[3], a[4], a[5]));
  return 0;
}
