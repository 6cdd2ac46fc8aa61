/* A plain C solver loop against the drop-in headers, as a CFD code calls libcfd2lcs: grid and
 * flags, one backward FTLE diagnostic, options, then cfd2lcs_update_c every step.  Built by
 * tests/test_c_driver.py with gcc -I include -I include/mpistub and linked against
 * libcfd2lcs_b200_dp.so.  Prints "ok <max|FTLE|>" on success, "error <message>" otherwise. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "cfd2lcs_inc_dp.h"
#include "cfd2lcs_b200.h"

#define NX 64
#define NY 32

int main(void) {
  const int n[3] = {NX, NY, 1}, offset[3] = {0, 0, 0};
  const int np = NX * NY;
  lcsdata_t *x = malloc(sizeof(lcsdata_t) * np), *y = malloc(sizeof(lcsdata_t) * np), *z = malloc(sizeof(lcsdata_t) * np);
  lcsdata_t *u = malloc(sizeof(lcsdata_t) * np), *v = malloc(sizeof(lcsdata_t) * np), *w = malloc(sizeof(lcsdata_t) * np);
  lcsdata_t *ftle = malloc(sizeof(lcsdata_t) * np);
  int *flag = malloc(sizeof(int) * np);
  for (int j = 0; j < NY; j++)
    for (int i = 0; i < NX; i++) {
      const int q = i + NX * j;
      x[q] = 2.0 * i / (NX - 1);
      y[q] = 1.0 * j / (NY - 1);
      z[q] = 0.0;
      flag[q] = (i == 0 || j == 0 || i == NX - 1 || j == NY - 1) ? LCS_SLIP : LCS_INTERNAL;
    }
  char label[LCS_NAMELEN] = "bkwd";
  cfd2lcs_init_c(MPI_COMM_WORLD, (int *)n, (int *)offset, x, y, z, flag);
  const int id = cfd2lcs_diagnostic_init_c(FTLE_BKWD, 0, 1.5, 0.15, label);
  cfd2lcs_set_option_c("INTEGRATOR", RK2);
  cfd2lcs_set_option_c("INTERPOLATOR", LINEAR);
  cfd2lcs_set_param_c("CFL", 0.5);
  const double pi = acos(-1.0), A = 0.1, eps = 0.25, om = 2.0 * pi / 10.0;
  for (int k = 0; k < 20; k++) {
    const double t = 0.1 * k, a = eps * sin(om * t), b = 1.0 - 2.0 * eps * sin(om * t);
    for (int q = 0; q < np; q++) {
      const double f = a * x[q] * x[q] + b * x[q], df = 2.0 * a * x[q] + b;
      u[q] = -pi * A * sin(pi * f) * cos(pi * y[q]);
      v[q] = pi * A * cos(pi * f) * sin(pi * y[q]) * df;
      w[q] = 0.0;
    }
    cfd2lcs_update_c((int *)n, u, v, w, t);
  }
  char msg[256];
  if (cfd2lcs_get_error_c(msg, sizeof msg)) {
    printf("error %s\n", msg);
    return 0;
  }
  if (cfd2lcs_get_ftle_c(id, ftle)) {
    printf("error no FTLE frame\n");
    return 0;
  }
  double mx = 0.0;
  for (int q = 0; q < np; q++) {
    if (!isfinite(ftle[q])) {
      printf("error non-finite FTLE\n");
      return 0;
    }
    mx = fmax(mx, fabs(ftle[q]));
  }
  cfd2lcs_finalize_c();
  printf("ok %.6e\n", mx);
  return 0;
}
