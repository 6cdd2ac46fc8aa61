/*
 * cfd2lcs_inc_sp.h -- user-level C interface of libcfd2lcs_b200, single precision build.
 *
 * Drop-in for the reference header of the same name (src/cfd2lcs_inc_single.h, installed
 * as include/cfd2lcs_inc_sp.h by the reference's src/Makefile:62-68).  Names, values and
 * prototypes are identical, so existing solvers compile unchanged; link against
 * libcfd2lcs_b200_sp.so instead of libcfd2lcs_sp.a.
 *
 * Extensions (finalize, error query, result access, device-pointer update) are declared in
 * cfd2lcs_b200.h; include it after this header.
 */
#ifndef CFD2LCS_INC_H
#define CFD2LCS_INC_H

#include <mpi.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Precision of the interface arrays (cfd2lcs_inc_single.h:17) */
typedef float lcsdata_t;

/* The string namelength (:22) */
#define LCS_NAMELEN 128

/* Boundary Condition Flags (:27-33) */
#define LCS_INTERNAL 0
#define LCS_INFLOW 1
#define LCS_OUTFLOW 2
#define LCS_WALL 3
#define LCS_SLIP 4
#define LCS_2D 5
#define LCS_MASK 6

/* LCS diagnostic types (:38-40) */
#define FTLE_FWD 0
#define FTLE_BKWD 1
#define LP_TRACER 2

/* Integration methods (:45-49) */
#define EULER 0
#define TRAPEZOIDAL 1
#define RK2 2
#define RK3 3
#define RK4 4

/* Interpolation methods (:54-59) */
#define NEAREST_NBR 0
#define LINEAR 1
#define QUADRATIC 2
#define CUBIC 3
#define TSE 5
#define TSE_LIMIT 6

/* True/False indicators (:64-65) */
#define LCS_FALSE 0
#define LCS_TRUE 1

/* Replaces cfd2lcs_init_c, src/cfd2lcs_c.c:67-83.  One MPI rank per library instance:
 * the communicator is accepted and ignored (offsets are normalised to 0). */
void cfd2lcs_init_c(MPI_Comm usercomm, int n[3], int offset[3], lcsdata_t *x, lcsdata_t *y, lcsdata_t *z, int *flag);

/* Replaces cfd2lcs_diagnostic_init_c, src/cfd2lcs_c.c:86-99.  Returns the handle. */
int cfd2lcs_diagnostic_init_c(int lcs_type, int resolution, lcsdata_t t, lcsdata_t h, char label[]);

/* Replaces cfd2lcs_update_c, src/cfd2lcs_c.c:102-115.  u, v, w are host arrays of
 * n[0]*n[1]*n[2] values, i fastest. */
void cfd2lcs_update_c(int n[3], lcsdata_t *u, lcsdata_t *v, lcsdata_t *w, lcsdata_t time);

/* Replaces cfd2lcs_diagnostic_destroy_c, src/cfd2lcs_c.c:118-122 (a no-op in the reference). */
void cfd2lcs_diagnostic_destroy_c(int lcs_handle);

/* Replaces cfd2lcs_set_option_c, src/cfd2lcs_c.c:125-132. */
void cfd2lcs_set_option_c(char option[], int val);

/* Replaces cfd2lcs_set_param_c, src/cfd2lcs_c.c:135-142. */
void cfd2lcs_set_param_c(char option[], lcsdata_t val);

#ifdef __cplusplus
}
#endif

#endif
