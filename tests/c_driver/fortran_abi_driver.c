/* The gfortran calling convention against libcfd2lcs_b200_dp.so: a Fortran solver's
 *   call cfd2lcs_init(comm, n, offset, x, y, z, flag)
 *   call cfd2lcs_diagnostic_init(id, FTLE_BKWD, 0, T, h, label)
 *   call cfd2lcs_set_option('INTEGRATOR', RK3)  ...
 * reaches the library as the external symbols cfd2lcs_*_ with every argument by reference and
 * one hidden trailing size_t length per CHARACTER argument, the string blank-padded and not
 * NUL-terminated (src/cfd2lcs.f90:2, 252, 436, 624; the reference's own C shim passes the same
 * calls, src/cfd2lcs_c.c:67-142).  This driver declares those prototypes itself, as the compiler
 * would, runs a 3-D flow with an option, a parameter and a label given that way, and the same
 * run through the cfd2lcs_*_c entry points, selected by argv[1] ("fortran" or "c").  It writes
 * the FTLE field of the last frame to argv[2] (raw doubles) and prints "ok" or "error <msg>".
 * Built and run by tests/test_fortran_abi.py. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cfd2lcs_inc_dp.h"
#include "cfd2lcs_b200.h"

/* gfortran's view of the external subroutines (no header of the library is used for these) */
void cfd2lcs_init_(int *comm, int *n, int *offset, double *x, double *y, double *z, int *flag);
void cfd2lcs_diagnostic_init_(int *id, int *type, int *res, double *T, double *h, char *label, size_t label_len);
void cfd2lcs_update_(int *n, double *u, double *v, double *w, double *time);
void cfd2lcs_set_option_(char *option, int *val, size_t len);
void cfd2lcs_set_param_(char *param, double *val, size_t len);
void cfd2lcs_diagnostic_destroy_(int *id);
void cfd2lcs_finalize_(void);

#define N 14

/* a CHARACTER(len) actual argument: blank-padded to len, no terminating NUL */
static char *fchar(const char *s, size_t len) {
  char *b = malloc(len);
  memset(b, ' ', len);
  memcpy(b, s, strlen(s));
  return b;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const int fortran = strcmp(argv[1], "fortran") == 0;
  int n[3] = {N, N, N}, offset[3] = {0, 0, 0};
  const int np = N * N * N;
  double *x = malloc(sizeof(double) * np), *y = malloc(sizeof(double) * np), *z = malloc(sizeof(double) * np);
  double *u = malloc(sizeof(double) * np), *v = malloc(sizeof(double) * np), *w = malloc(sizeof(double) * np);
  double *ftle = malloc(sizeof(double) * np);
  int *flag = malloc(sizeof(int) * np);
  const double pi = acos(-1.0), L = 2.0 * pi;
  for (int k = 0; k < N; k++)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < N; i++) {
        const int q = i + N * (j + N * k);
        x[q] = (i + 0.5) * L / N;
        y[q] = (j + 0.5) * L / N;
        z[q] = (k + 0.5) * L / N;
        flag[q] = LCS_INTERNAL;
      }
  int id = -1;
  double T = 0.6, h = 0.2;
  if (fortran) {
    int comm = 0, type = FTLE_BKWD, res = 0, rk3 = RK3, cubic = CUBIC;
    double cfl = 0.4;
    char *label = fchar("abc_bkwd", 32), *o1 = fchar("INTEGRATOR", 24), *o2 = fchar("INTERPOLATOR", 20), *p1 = fchar("CFL", 12);
    cfd2lcs_init_(&comm, n, offset, x, y, z, flag);
    cfd2lcs_diagnostic_init_(&id, &type, &res, &T, &h, label, 32);
    cfd2lcs_set_option_(o1, &rk3, 24);
    cfd2lcs_set_option_(o2, &cubic, 20);
    cfd2lcs_set_param_(p1, &cfl, 12);
  } else {
    char label[LCS_NAMELEN] = "abc_bkwd";
    cfd2lcs_init_c(MPI_COMM_WORLD, n, offset, x, y, z, flag);
    id = cfd2lcs_diagnostic_init_c(FTLE_BKWD, 0, T, h, label);
    cfd2lcs_set_option_c("INTEGRATOR", RK3);
    cfd2lcs_set_option_c("INTERPOLATOR", CUBIC);
    cfd2lcs_set_param_c("CFL", 0.4);
  }
  const double A = sqrt(3.0), B = sqrt(2.0), C = 1.0;
  for (int step = 0; step < 14; step++) {
    double t = 0.05 * step;
    for (int q = 0; q < np; q++) {
      const double s = 1.0 + 0.3 * sin(t);
      u[q] = s * (A * sin(z[q]) + C * cos(y[q]));
      v[q] = s * (B * sin(x[q]) + A * cos(z[q]));
      w[q] = s * (C * sin(y[q]) + B * cos(x[q]));
    }
    if (fortran) cfd2lcs_update_(n, u, v, w, &t);
    else cfd2lcs_update_c(n, u, v, w, t);
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
  FILE *f = fopen(argv[2], "wb");
  if (!f || fwrite(ftle, sizeof(double), np, f) != (size_t)np) {
    printf("error cannot write %s\n", argv[2]);
    return 0;
  }
  fclose(f);
  if (fortran) {
    cfd2lcs_diagnostic_destroy_(&id);
    cfd2lcs_finalize_();
  } else {
    cfd2lcs_diagnostic_destroy_c(id);
    cfd2lcs_finalize_c();
  }
  printf("ok %d\n", id);
  return 0;
}
