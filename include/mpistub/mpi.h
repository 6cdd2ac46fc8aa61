/*
 * Single-rank stand-in for <mpi.h>, for solvers built without MPI.  libcfd2lcs_b200 runs
 * one rank per library instance and never calls MPI, so the interface header only needs
 * the MPI_Comm type.  Put this directory on the include path ONLY when no MPI is used;
 * with a real MPI, compile against that MPI's mpi.h instead.
 */
#ifndef CFD2LCS_B200_MPI_STUB_H
#define CFD2LCS_B200_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Fint;
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#define MPI_SUCCESS 0
static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }
#endif
