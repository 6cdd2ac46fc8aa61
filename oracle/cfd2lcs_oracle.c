/*
 * cfd2lcs_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * A CPU restatement of libcfd2lcs's FTLE hot path as it behaves on ONE MPI rank:
 * grid ingest, ghost/boundary padding, CFL subcycling, the backward semi-Lagrangian
 * flow-map update, the forward particle update, the in-memory sub-flow-map ring,
 * the composition (reconstruct) and the FTLE.  Every routine names the reference
 * file:line it restates (paths relative to the libcfd2lcs source tree).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * may load this library.  The shipped library (libcfd2lcs_b200) never links it.
 *
 * PARITY UNPINNED: the reference ships no tests, no golden vectors and no fixtures,
 * and it cannot be compiled here (it needs gfortran, MPI and LAPACK, none of which are
 * installed).  This restatement is therefore checked against analytic known answers
 * (translation, rigid rotation, polynomial reproduction of the spline) rather than
 * against outputs of the reference itself.
 *
 * Build: oracle/Makefile -> liboracle_dp.so (real = double, the reference's "dp"
 * build) and liboracle_sp.so (real = float, the "sp" build).  Compiled without FMA
 * contraction, as gfortran -O3 compiles the reference for baseline x86-64.
 *
 * Deliberate single-rank simplifications (all identities when nprocs == 1):
 *   - every MPI collective is the identity; exchange_sdata reduces to the SELF copies
 *     of src/comms_m.f90:814-822; exchange_lp_alltoall / exchange_lpmap keep particle
 *     order (pack order == unpack order for one rank);
 *   - the cfd2lcs_tmp/ sub-flow-map files become an in-memory ring (a fresh, empty
 *     temp directory is assumed at init);
 *   - no output files are written (write_lcs is out of scope).
 */
#include <math.h>
#include <float.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_SP
typedef float real;
#define R_TINY FLT_MIN
#define R_HUGE FLT_MAX
#else
typedef double real;
#define R_TINY DBL_MIN
#define R_HUGE DBL_MAX
#endif

/* cfd2lcs_inc_double.h:27-65 */
enum { LCS_INTERNAL = 0, LCS_INFLOW = 1, LCS_OUTFLOW = 2, LCS_WALL = 3, LCS_SLIP = 4, LCS_2D = 5, LCS_MASK = 6 };
enum { FTLE_FWD = 0, FTLE_BKWD = 1, LP_TRACER = 2 };
enum { EULER = 0, TRAPEZOIDAL = 1, RK2 = 2, RK3 = 3, RK4 = 4 };
enum { NEAREST_NBR = 0, LINEAR = 1, QUADRATIC = 2, CUBIC = 3, TSE = 5, TSE_LIMIT = 6 };
enum { LCS_FALSE = 0, LCS_TRUE = 1 };
/* data_m.f90:110-121 */
enum { LP_IB = -1, LP_UNKNOWN = -2, LP_RECYCLE = -3, LP_STICK = -4 };
enum { FWD = 1, BKWD = -1 };
enum { NO_COMM = 0, SELF_COMM = 1 };

/* Neighbour offsets, data_m.f90:124-152 (order matters for tracking ties). */
static const int NBR[27][3] = {
    {0, 0, 0},   {-1, 0, 0},  {0, -1, 0}, {0, 0, -1}, {1, 0, 0},  {0, 1, 0},  {0, 0, 1},
    {-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {-1, 0, -1}, {1, 0, -1}, {-1, 1, -1}, {0, 1, -1},
    {1, 1, -1},  {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0}, {1, 1, 0},  {-1, -1, 1}, {0, -1, 1},
    {1, -1, 1},  {-1, 0, 1},  {1, 0, 1},   {-1, 1, 1}, {0, 1, 1},  {1, 1, 1}};

#define MAXLCS 64
#define MAXVSTEP 4096
#define MAXMSG 512

/* ------------------------------------------------------------------------------------
 * Ghost-padded structured storage: Fortran bounds (0:n+1) in each direction, i fastest
 * (structured_m.f90:73-96; NGHOST_CFD = 1, data_m.f90:106).
 * ------------------------------------------------------------------------------------ */
typedef struct {
    int ni, nj, nk;
    long sx, sy, ntot;
} dims_t;

static inline long PX(const dims_t *d, int i, int j, int k) { return (long)i + d->sx * (long)j + d->sy * (long)k; }

typedef struct {
    real *c[3];
} sr1_t;

typedef struct sgrid_s {
    /* dimensions (one rank: local == global, offsets 0) */
    dims_t d;
    int gn[3];
    int per[3];
    int rectilinear;
    sr1_t grid;
    int *bcflag;
    sr1_t bcnorm;
    real ps[3][3][3][3]; /* periodic_shift(i,j,k,c) stored [k+1][j+1][i+1][c] */
    real bb[6];
    int scomm_flag[3][3][3]; /* max-connectivity SELF/NO comm flag per direction */
    /* non-rectilinear grids: least-squares gradient weights of the six face neighbours
     * (compute_lsgw with full_conn = .false., sgrid_m.f90:421-424; nbr = 2..7 of NBR_OFFSET,
     * stored at [nbr-2][component], padded, zero on the ghost layer), and the positions of
     * the smallest / largest coordinate (minloc / maxloc over the padded arrays, counted from
     * 1 as Fortran returns them) for the node guess of exchange_lp_alltoall */
    real *lsw[6][3];
    real ijk_min[3][3], ijk_max[3][3]; /* [coordinate][direction] */
} sgrid_t;

typedef struct {
    int np;
    int direction;
    int recursive_tracking;
    real dt_factor;
    real *xp[3], *up[3], *dx[3];
    int *no[3], *no_scfd[3];
    int *flag;
    sr1_t fm;
    real lifetime; /* time advected (integrate_lp, lp_motion_m.f90:332) */
    const struct sgrid_s *sg; /* lp%sgrid: the grid of the particle set (the lcs grid) */
} lp_t;

typedef struct lcs_s {
    int id;
    int diagnostic;
    real T, h;
    lp_t lp;
    real *ftle; /* padded sr0 */
    real *inv[5]; /* velocity invariants Q, D, C, H, L2 of the last frame (padded sr0) */
    real *l2margin; /* checker aid: middle eigenvalue / largest magnitude (how close L2 is to a tie) */
    sr1_t fm_out; /* composed flow map of the last FTLE frame (written by write_lcs) */
    char label[136]; /* lcs%label, trimmed */
    int dead;        /* an LP_TRACER set that was never injected or outlived T (destroy_lcs) */
    sgrid_t *sg;     /* lcs%sgrid: the solver grid (resolution 0) or its own refined copy */
    int own_sg;
    struct lcs_s *aux[6]; /* AUX_GRID particle sets X0, Y0, Z0, X1, Y1, Z1 (lcs%lpX0 ...) */
    int naux;
    int nslot;
    real **slot[3]; /* slot[c][s] -> interior values of stored sub-flow map */
    int *written;
} lcs_t;

static struct {
    int error;
    char msg[MAXMSG];
    /* options (data_m.f90:19-92) */
    int integrator, interpolator, incompressible, aux_grid, velocity_invariants;
    real cfl_max;
    /* state */
    int inited;
    sgrid_t g;
    sr1_t u_n, u_np1, delta;
    real t_n, t_np1;
    int first_call;
    int nlcs;
    lcs_t *lcs[MAXLCS];
    long long integrations_fwd, integrations_bkwd;
    int last_nsub_fwd, last_nsub_bkwd;
    long long ftle_frames;
    /* velocity snapshots by ring step (the cfd2lcs_tmp/<rank>_<u label>_<step> files of
     * write_flowmap_substep, flowmap_m.f90:139-151): one set shared by every diagnostic,
     * interior values; steps 0 .. NVSTEP-1 */
    real *vring[3][MAXVSTEP];
    int vwritten[MAXVSTEP];
    /* output files (write_lcs): WRITE_LCS switches them on; FLOWMAP_IO and VELOCITY_IO
     * default to TRUE (data_m.f90:44-49), kept here as their negations so that zeroed state
     * means the defaults */
    int write_lcs, no_flowmap_io, no_velocity_io, bcflag_io;
    /* TRACER_INJECT_X/Y/Z/RADIUS (data_m.f90:86-89: the centre defaults to huge(1.0), the
     * radius to 0); tracer_set marks the ones given */
    real tracer_c[3], tracer_r;
    int tracer_set[3];
    char outdir[512];
} S = {0, "", RK2, LINEAR, 0, 0, 0, (real)0.5, 0};

static void latch(const char *m) {
    if (!S.error) snprintf(S.msg, MAXMSG, "%s", m);
    S.error = 1;
}

static real *zalloc(long n) {
    real *p = (real *)calloc((size_t)(n > 0 ? n : 1), sizeof(real));
    if (!p) {
        latch("oracle: out of host memory");
    }
    return p;
}

static void sr1_alloc(sr1_t *a, const dims_t *d) {
    for (int c = 0; c < 3; c++) a->c[c] = zalloc(d->ntot);
}
static void sr1_free(sr1_t *a) {
    for (int c = 0; c < 3; c++) {
        free(a->c[c]);
        a->c[c] = NULL;
    }
}

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline real rmax(real a, real b) { return a > b ? a : b; }
static inline real rmin(real a, real b) { return a < b ? a : b; }

/* Fortran NINT: round half away from zero. */
static inline int fnint(real v) { return (int)(v >= 0 ? floor((double)v + 0.5) : -floor(-(double)v + 0.5)); }

/* ------------------------------------------------------------------------------------
 * exchange_sdata on one rank (comms_m.f90:679-869 with the SELF copy at :814-822).
 * For every direction d (26 for max connectivity, 6 for face) whose neighbour is SELF
 * (all non-zero components periodic, comms_m.f90:241-279), the interior slab next to
 * face d is copied to the ghost slab on the opposite side.  Coordinates carry the
 * periodic shift of d, with the z component read at (i,k,k) as comms_m.f90:750 does.
 * ------------------------------------------------------------------------------------ */
static int comm_self(const sgrid_t *g, int di, int dj, int dk) {
    if (di && !g->per[0]) return 0;
    if (dj && !g->per[1]) return 0;
    if (dk && !g->per[2]) return 0;
    return 1;
}

static void exchange_self(const sgrid_t *g, real *const *f, int ncomp, int max_conn, int translate) {
    const dims_t *d = &g->d;
    int n[3] = {d->ni, d->nj, d->nk};
    int ncomm = max_conn ? 27 : 7;
    for (int ic = 1; ic < ncomm; ic++) {
        int dd[3] = {NBR[ic][0], NBR[ic][1], NBR[ic][2]};
        if (!comm_self(g, dd[0], dd[1], dd[2])) continue;
        int lo[3], hi[3];
        for (int a = 0; a < 3; a++) {
            /* pack_list (comms_m.f90:357-415): d=-1 -> [1,ng], 0 -> [1,n], 1 -> [n-ng+1,n] */
            if (dd[a] == -1) { lo[a] = 1; hi[a] = 1; }
            else if (dd[a] == 0) { lo[a] = 1; hi[a] = n[a]; }
            else { lo[a] = n[a]; hi[a] = n[a]; }
        }
        real sh[3] = {0, 0, 0};
        if (translate) {
            sh[0] = g->ps[dd[2] + 1][dd[1] + 1][dd[0] + 1][0];
            sh[1] = g->ps[dd[2] + 1][dd[1] + 1][dd[0] + 1][1];
            sh[2] = g->ps[dd[2] + 1][dd[2] + 1][dd[0] + 1][2]; /* (i,k,k): comms_m.f90:750 */
        }
        for (int k = lo[2]; k <= hi[2]; k++)
            for (int j = lo[1]; j <= hi[1]; j++)
                for (int i = lo[0]; i <= hi[0]; i++) {
                    /* ghost on the opposite side: q = p - d*n */
                    int qi = i - dd[0] * n[0], qj = j - dd[1] * n[1], qk = k - dd[2] * n[2];
                    long src = PX(d, i, j, k), dst = PX(d, qi, qj, qk);
                    for (int c = 0; c < ncomp; c++) f[c][dst] = f[c][src] + sh[c];
                }
    }
}

/* ------------------------------------------------------------------------------------
 * init_sgrid (sgrid_m.f90:16-444), one rank.
 * ------------------------------------------------------------------------------------ */
static void cross_unit(const real v1[3], const real v2[3], real out[3]) {
    /* geometry_m.f90:12-31 (unitvector = .true.) */
    out[0] = v1[1] * v2[2] - v1[2] * v2[1];
    out[1] = v1[2] * v2[0] - v1[0] * v2[2];
    out[2] = v1[0] * v2[1] - v1[1] * v2[0];
    real m = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    if (m > 0) {
        out[0] /= m; out[1] /= m; out[2] /= m;
    }
}

static void check_rectilinear(sgrid_t *g) {
    /* sgrid_m.f90:868-949 (including the z loop's 1:k with k = nk+1 left over) */
    const dims_t *d = &g->d;
    int ni = d->ni, nj = d->nj, nk = d->nk;
    const real TOL = (real)1e-4f; /* real(LCSRP),parameter:: TOL = 1e-4, a default-real literal */
    real mx[3], mn[3];
    for (int c = 0; c < 3; c++) { mx[c] = -R_HUGE; mn[c] = R_HUGE; }
    for (long p = 0; p < d->ntot; p++)
        for (int c = 0; c < 3; c++) {
            mx[c] = rmax(mx[c], g->grid.c[c][p]);
            mn[c] = rmin(mn[c], g->grid.c[c][p]);
        }
    real big = rmax(rmax(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
    int ortho[3] = {1, 1, 1};
    /* x lines */
    for (int k = 1; k <= nk && ortho[0]; k++)
        for (int j = 1; j <= nj && ortho[0]; j++) {
            real a[3] = {-R_HUGE, -R_HUGE, -R_HUGE}, b[3] = {R_HUGE, R_HUGE, R_HUGE};
            for (int i = 1; i <= ni; i++)
                for (int c = 0; c < 3; c++) {
                    real v = g->grid.c[c][PX(d, i, j, k)];
                    a[c] = rmax(a[c], v); b[c] = rmin(b[c], v);
                }
            if (fabs(a[1] - b[1]) / big > TOL || fabs(a[2] - b[2]) / big > TOL) ortho[0] = 0;
        }
    for (int k = 1; k <= nk && ortho[1]; k++)
        for (int i = 1; i <= ni && ortho[1]; i++) {
            real a[3] = {-R_HUGE, -R_HUGE, -R_HUGE}, b[3] = {R_HUGE, R_HUGE, R_HUGE};
            for (int j = 1; j <= nj; j++)
                for (int c = 0; c < 3; c++) {
                    real v = g->grid.c[c][PX(d, i, j, k)];
                    a[c] = rmax(a[c], v); b[c] = rmin(b[c], v);
                }
            if (fabs(a[0] - b[0]) / big > TOL || fabs(a[2] - b[2]) / big > TOL) ortho[1] = 0;
        }
    for (int j = 1; j <= nj && ortho[2]; j++)
        for (int i = 1; i <= ni && ortho[2]; i++) {
            real a[3] = {-R_HUGE, -R_HUGE, -R_HUGE}, b[3] = {R_HUGE, R_HUGE, R_HUGE};
            for (int k = 1; k <= nk + 1; k++)
                for (int c = 0; c < 3; c++) {
                    real v = g->grid.c[c][PX(d, i, j, k)];
                    a[c] = rmax(a[c], v); b[c] = rmin(b[c], v);
                }
            if (fabs(a[0] - b[0]) / big > TOL || fabs(a[1] - b[1]) / big > TOL) ortho[2] = 0;
        }
    g->rectilinear = ortho[0] && ortho[1] && ortho[2];
}

/* compute_lsgw (gradient_m.f90:114-217) at interior node (i,j,k) for the neighbours
 * nb = first..last of NBR_OFFSET: inverse-distance weights and the closed-form solution of
 * the 3x3 least-squares system, w[nb][c].  Products and sums in the reference's order:
 * sum(dx(1:3)**2) and idw*dx(a)**2 form the squares first; sdenom subtracts s*(t**2). */
static void lsq_weights(const sgrid_t *g, int i, int j, int k, int first, int last, real w[27][3]) {
    const dims_t *d = &g->d;
    const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
    long p = PX(d, i, j, k);
    real sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    for (int nb = first; nb <= last; nb++) {
        long q = PX(d, i + NBR[nb][0], j + NBR[nb][1], k + NBR[nb][2]);
        real dx0 = X[q] - X[p], dx1 = Y[q] - Y[p], dx2 = Z[q] - Z[p];
        real idw = (real)1 / (dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
        sxx = sxx + idw * (dx0 * dx0);
        syy = syy + idw * (dx1 * dx1);
        szz = szz + idw * (dx2 * dx2);
        sxy = sxy + idw * dx0 * dx1;
        sxz = sxz + idw * dx0 * dx2;
        syz = syz + idw * dx1 * dx2;
    }
    real sden = (real)2 * sxy * sxz * syz + sxx * syy * szz - sxx * (syz * syz) - syy * (sxz * sxz) - szz * (sxy * sxy);
    for (int nb = first; nb <= last; nb++) {
        long q = PX(d, i + NBR[nb][0], j + NBR[nb][1], k + NBR[nb][2]);
        real dx0 = X[q] - X[p], dx1 = Y[q] - Y[p], dx2 = Z[q] - Z[p];
        real idw = (real)1 / (dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
        w[nb][0] = idw * ((syy * szz - syz * syz) * dx0 + (sxz * syz - sxy * szz) * dx1 + (sxy * syz - sxz * syy) * dx2) / sden;
        w[nb][1] = idw * ((sxz * syz - sxy * szz) * dx0 + (sxx * szz - sxz * sxz) * dx1 + (sxy * sxz - syz * sxx) * dx2) / sden;
        w[nb][2] = idw * ((sxy * syz - sxz * syy) * dx0 + (sxy * sxz - syz * sxx) * dx1 + (sxx * syy - sxy * sxy) * dx2) / sden;
    }
}

static void compute_bcnorm(sgrid_t *g) {
    /* sgrid_m.f90:385-419 with compute_lsgw(full_conn) gradient_m.f90:114-217 and
     * grad_sr0_ls gradient_m.f90:297-335 */
    const dims_t *d = &g->d;
    real *bc = zalloc(d->ntot);
    for (int k = 0; k <= d->nk + 1; k++)
        for (int j = 0; j <= d->nj + 1; j++)
            for (int i = 0; i <= d->ni + 1; i++) {
                long p = PX(d, i, j, k);
                int f = g->bcflag[p];
                bc[p] = (f == LCS_2D) ? (real)LCS_INTERNAL : (real)imin(f, 1);
            }
    exchange_self(g, &bc, 1, 1, 0);
    sr1_alloc(&g->bcnorm, d);
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long p = PX(d, i, j, k);
                real w[27][3];
                lsq_weights(g, i, j, k, 1, 26, w);
                real gx = 0, gy = 0, gz = 0;
                for (int nb = 1; nb < 27; nb++) {
                    long q = PX(d, i + NBR[nb][0], j + NBR[nb][1], k + NBR[nb][2]);
                    real df = bc[q] - bc[p];
                    gx = gx + df * w[nb][0];
                    gy = gy + df * w[nb][1];
                    gz = gz + df * w[nb][2];
                }
                real mag = gx * gx + gy * gy + gz * gz;
                if (mag <= 0) {
                    gx = gy = gz = 0;
                } else {
                    gx = gx / sqrt(mag); gy = gy / sqrt(mag); gz = gz / sqrt(mag);
                }
                g->bcnorm.c[0][p] = gx; g->bcnorm.c[1][p] = gy; g->bcnorm.c[2][p] = gz;
            }
    free(bc);
}

/* Non-rectilinear grids (sgrid_m.f90:421-424): the face-neighbour least-squares weights, and
 * minloc / maxloc of each coordinate for exchange_lp_alltoall's node guess
 * (comms_m.f90:1625-1632). */
static void compute_lsgw_face(sgrid_t *g) {
    const dims_t *d = &g->d;
    for (int nb = 0; nb < 6; nb++)
        for (int c = 0; c < 3; c++) g->lsw[nb][c] = zalloc(d->ntot);
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                real w[27][3];
                lsq_weights(g, i, j, k, 1, 6, w);
                long p = PX(d, i, j, k);
                for (int nb = 1; nb <= 6; nb++)
                    for (int c = 0; c < 3; c++) g->lsw[nb - 1][c][p] = w[nb][c];
            }
    for (int c = 0; c < 3; c++) {
        /* the first position in array element order (i fastest) holding the extreme value */
        long pmin = 0, pmax = 0;
        for (long p = 1; p < d->ntot; p++) {
            if (g->grid.c[c][p] < g->grid.c[c][pmin]) pmin = p;
            if (g->grid.c[c][p] > g->grid.c[c][pmax]) pmax = p;
        }
        const long pp[2] = {pmin, pmax};
        for (int e = 0; e < 2; e++) {
            long p = pp[e];
            real pos[3] = {(real)(p % d->sx + 1), (real)((p / d->sx) % (d->nj + 2) + 1), (real)(p / d->sy + 1)};
            for (int a = 0; a < 3; a++) {
                if (e == 0) g->ijk_min[c][a] = pos[a];
                else g->ijk_max[c][a] = pos[a];
            }
        }
    }
}

/* grad_sr1_ls / grad_sr0_ls (gradient_m.f90:241-335) of one component at padded node p:
 * sum over the face neighbours of (f(nbr) - f(p)) * weight; zero on the ghost layer */
static void grad_ls(const sgrid_t *g, const real *F, int i, int j, int k, real gr[3]) {
    const dims_t *d = &g->d;
    gr[0] = gr[1] = gr[2] = 0;
    if (i < 1 || j < 1 || k < 1 || i > d->ni || j > d->nj || k > d->nk) return;
    long p = PX(d, i, j, k);
    for (int nb = 1; nb <= 6; nb++) {
        long q = PX(d, i + NBR[nb][0], j + NBR[nb][1], k + NBR[nb][2]);
        real df = F[q] - F[p];
        gr[0] = gr[0] + df * g->lsw[nb - 1][0][p];
        gr[1] = gr[1] + df * g->lsw[nb - 1][1][p];
        gr[2] = gr[2] + df * g->lsw[nb - 1][2][p];
    }
}

static int init_sgrid(sgrid_t *g, const int n[3], const real *x, const real *y, const real *z, const int *flag) {
    dims_t *d = &g->d;
    d->ni = n[0]; d->nj = n[1]; d->nk = n[2];
    if (d->ni < 1 || d->nj < 1 || d->nk < 1) {
        latch("init: ng > ni, nj or nk");
        return 1;
    }
    d->sx = d->ni + 2;
    d->sy = d->sx * (long)(d->nj + 2);
    d->ntot = d->sy * (long)(d->nk + 2);
    int ni = d->ni, nj = d->nj, nk = d->nk;
    for (int a = 0; a < 3; a++) g->gn[a] = n[a];
    /* periodicity from flags, sgrid_m.f90:107-136 */
    int pl[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++)
            for (int i = 0; i < ni; i++) {
                int f = flag[i + (long)ni * (j + (long)nj * k)];
                if (f != LCS_INTERNAL) continue;
                if (i == 0) pl[0] = 1;
                if (j == 0) pl[1] = 1;
                if (k == 0) pl[2] = 1;
                if (i == ni - 1) pl[3] = 1;
                if (j == nj - 1) pl[4] = 1;
                if (k == nk - 1) pl[5] = 1;
            }
    for (int a = 0; a < 3; a++)
        if (pl[a] != pl[a + 3]) {
            latch("init: periodicity does not appear to match; check flag values passed to cfd2lcs_init");
            return 1;
        }
    for (int a = 0; a < 3; a++) g->per[a] = pl[a] && g->gn[a] != 1;

    sr1_alloc(&g->grid, d);
    g->bcflag = (int *)calloc((size_t)d->ntot, sizeof(int));
    /* interior, sgrid_m.f90:169-178 */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                long s = (i - 1) + (long)ni * ((j - 1) + (long)nj * (k - 1));
                long p = PX(d, i, j, k);
                g->grid.c[0][p] = x[s]; g->grid.c[1][p] = y[s]; g->grid.c[2][p] = z[s];
                g->bcflag[p] = flag[s];
            }
    /* fake (mirrored) ghost coordinates and ghost flags, sgrid_m.f90:182-214 */
    for (int k = 0; k <= nk + 1; k++)
        for (int j = 0; j <= nj + 1; j++)
            for (int i = 0; i <= ni + 1; i++) {
                int ib = clampi(i, 1, ni), jb = clampi(j, 1, nj), kb = clampi(k, 1, nk);
                if (i == ib && j == jb && k == kb) continue;
                int iib = clampi(ib + (ib - i), 1, ni), jib = clampi(jb + (jb - j), 1, nj), kib = clampi(kb + (kb - k), 1, nk);
                long pb = PX(d, ib, jb, kb), pib = PX(d, iib, jib, kib), p = PX(d, i, j, k);
                for (int c = 0; c < 3; c++) {
                    real delta = g->grid.c[c][pb] - g->grid.c[c][pib];
                    g->grid.c[c][p] = g->grid.c[c][pb] + delta;
                }
                g->bcflag[p] = g->bcflag[pb];
            }
    /* singleton directions, sgrid_m.f90:217-255 */
    if (g->gn[0] == 1)
        for (int k = 0; k <= nk + 1; k++)
            for (int j = 0; j <= nj + 1; j++) {
                int f1 = g->bcflag[PX(d, 1, j, k)];
                int v = (f1 == LCS_INTERNAL) ? LCS_2D : f1;
                g->bcflag[PX(d, 0, j, k)] = v;
                for (int i = 2; i <= ni + 1; i++) g->bcflag[PX(d, i, j, k)] = v;
            }
    if (g->gn[1] == 1)
        for (int k = 0; k <= nk + 1; k++)
            for (int i = 0; i <= ni + 1; i++) {
                int f1 = g->bcflag[PX(d, i, 1, k)];
                int v = (f1 == LCS_INTERNAL) ? LCS_2D : f1;
                g->bcflag[PX(d, i, 0, k)] = v;
                for (int j = 2; j <= nj + 1; j++) g->bcflag[PX(d, i, j, k)] = v;
            }
    if (g->gn[2] == 1)
        for (int j = 0; j <= nj + 1; j++)
            for (int i = 0; i <= ni + 1; i++) {
                int f1 = g->bcflag[PX(d, i, j, 1)];
                int v = (f1 == LCS_INTERNAL) ? LCS_2D : f1;
                g->bcflag[PX(d, i, j, 0)] = v;
                for (int k = 2; k <= nk + 1; k++) g->bcflag[PX(d, i, j, k)] = v;
            }
    /* SELF/NO comm flags (comms_m.f90:241-279) */
    for (int dk = -1; dk <= 1; dk++)
        for (int dj = -1; dj <= 1; dj++)
            for (int di = -1; di <= 1; di++) g->scomm_flag[dk + 1][dj + 1][di + 1] = comm_self(g, di, dj, dk) ? SELF_COMM : NO_COMM;
    /* periodic shifts: exchange with zero shift, difference to the fakes, exchange again
     * (sgrid_m.f90:257-297) */
    sr1_t fake;
    sr1_alloc(&fake, d);
    for (int c = 0; c < 3; c++) memcpy(fake.c[c], g->grid.c[c], sizeof(real) * (size_t)d->ntot);
    memset(g->ps, 0, sizeof(g->ps));
    exchange_self(g, g->grid.c, 3, 1, 1);
    for (int c = 0; c < 3; c++)
        for (long p = 0; p < d->ntot; p++) fake.c[c][p] = g->grid.c[c][p] - fake.c[c][p];
    for (int kk = -1; kk <= 1; kk++)
        for (int jj = -1; jj <= 1; jj++)
            for (int ii = -1; ii <= 1; ii++) {
                int gi = ii == -1 ? 0 : (ii == 0 ? 1 : ni + 1);
                int gj = jj == -1 ? 0 : (jj == 0 ? 1 : nj + 1);
                int gk = kk == -1 ? 0 : (kk == 0 ? 1 : nk + 1);
                for (int c = 0; c < 3; c++) g->ps[kk + 1][jj + 1][ii + 1][c] = fake.c[c][PX(d, gi, gj, gk)];
            }
    exchange_self(g, g->grid.c, 3, 1, 1);
    sr1_free(&fake);
    /* 2-D extrusion of the singleton direction, sgrid_m.f90:304-359 */
    {
        real sc[3];
        for (int c = 0; c < 3; c++) {
            real a = -R_HUGE, b = R_HUGE;
            for (int k = 1; k <= nk; k++)
                for (int j = 1; j <= nj; j++)
                    for (int i = 1; i <= ni; i++) {
                        real v = g->grid.c[c][PX(d, i, j, k)];
                        a = rmax(a, v); b = rmin(b, v);
                    }
            sc[c] = a - b;
        }
        real scaling = rmax(rmax(sc[0], sc[1]), sc[2]) / (real)imax(imax(ni, nj), nk);
        const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
        real *Xw = g->grid.c[0], *Yw = g->grid.c[1], *Zw = g->grid.c[2];
        (void)X; (void)Y; (void)Z;
        for (int k = 0; k <= nk + 1; k++)
            for (int j = 0; j <= nj + 1; j++)
                for (int i = 0; i <= ni + 1; i++) {
                    int im1 = imax(i - 1, 0), ip1 = imin(i + 1, ni + 1);
                    int jm1 = imax(j - 1, 0), jp1 = imin(j + 1, nj + 1);
                    int km1 = imax(k - 1, 0), kp1 = imin(k + 1, nk + 1);
                    real dl[3] = {0, 0, 0}, v1[3], v2[3], cu[3];
                    if (g->gn[0] == 1 && i != 1) {
                        for (int c = 0; c < 3; c++) {
                            v1[c] = g->grid.c[c][PX(d, 1, jp1, 1)] - g->grid.c[c][PX(d, 1, jm1, 1)];
                            v2[c] = g->grid.c[c][PX(d, 1, 1, kp1)] - g->grid.c[c][PX(d, 1, 1, km1)];
                        }
                        cross_unit(v1, v2, cu);
                        for (int c = 0; c < 3; c++) dl[c] = (real)(i - 1) * cu[c];
                    }
                    if (g->gn[1] == 1 && j != 1) {
                        for (int c = 0; c < 3; c++) {
                            v1[c] = g->grid.c[c][PX(d, ip1, 1, 1)] - g->grid.c[c][PX(d, im1, 1, 1)];
                            v2[c] = g->grid.c[c][PX(d, 1, 1, kp1)] - g->grid.c[c][PX(d, 1, 1, km1)];
                        }
                        cross_unit(v1, v2, cu);
                        for (int c = 0; c < 3; c++) dl[c] = (real)(j - 1) * cu[c];
                    }
                    if (g->gn[2] == 1 && k != 1) {
                        for (int c = 0; c < 3; c++) {
                            v1[c] = g->grid.c[c][PX(d, ip1, 1, 1)] - g->grid.c[c][PX(d, im1, 1, 1)];
                            v2[c] = g->grid.c[c][PX(d, 1, jp1, 1)] - g->grid.c[c][PX(d, 1, jm1, 1)];
                        }
                        cross_unit(v1, v2, cu);
                        for (int c = 0; c < 3; c++) dl[c] = (real)(k - 1) * cu[c];
                    }
                    long p = PX(d, i, j, k);
                    Xw[p] = Xw[p] + dl[0] * scaling;
                    Yw[p] = Yw[p] + dl[1] * scaling;
                    Zw[p] = Zw[p] + dl[2] * scaling;
                }
    }
    /* bounding box including ghosts, sgrid_m.f90:362-372 */
    for (int c = 0; c < 3; c++) {
        real a = R_HUGE, b = -R_HUGE;
        for (long p = 0; p < d->ntot; p++) {
            a = rmin(a, g->grid.c[c][p]);
            b = rmax(b, g->grid.c[c][p]);
        }
        g->bb[c] = a;
        g->bb[c + 3] = b;
    }
    check_rectilinear(g);
    compute_bcnorm(g);
    if (!g->rectilinear) compute_lsgw_face(g);
    return 0;
}

/* compute_delta_xyz, sgrid_m.f90:951-1014: 1/(half span of the 3x3x3 neighbourhood) */
static void compute_delta(const sgrid_t *g, sr1_t *delta) {
    const dims_t *d = &g->d;
    sr1_alloc(delta, d);
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                for (int c = 0; c < 3; c++) {
                    real a = -R_HUGE, b = R_HUGE;
                    for (int kk = k - 1; kk <= k + 1; kk++)
                        for (int jj = j - 1; jj <= j + 1; jj++)
                            for (int ii = i - 1; ii <= i + 1; ii++) {
                                real v = g->grid.c[c][PX(d, ii, jj, kk)];
                                a = rmax(a, v); b = rmin(b, v);
                            }
                    real dl = (real)0.5 * fabs(a - b);
                    delta->c[c][PX(d, i, j, k)] = dl > 0 ? (real)1 / dl : (real)0;
                }
            }
}

/* ------------------------------------------------------------------------------------
 * Boundary conditions on padded fields.
 * ------------------------------------------------------------------------------------ */
/* set_velocity_bc, sgrid_m.f90:810-866 */
static void set_velocity_bc(const sgrid_t *g, sr1_t *v) {
    const dims_t *d = &g->d;
    for (int k = 0; k <= d->nk + 1; k++)
        for (int j = 0; j <= d->nj + 1; j++)
            for (int i = 0; i <= d->ni + 1; i++) {
                long p = PX(d, i, j, k);
                int f = g->bcflag[p];
                int inside = i >= 1 && j >= 1 && k >= 1 && i <= d->ni && j <= d->nj && k <= d->nk;
                switch (f) {
                case LCS_INTERNAL: break;
                case LCS_MASK:
                    for (int c = 0; c < 3; c++) v->c[c][p] = 0;
                    break;
                case LCS_WALL:
                    if (inside) break;
                    for (int c = 0; c < 3; c++) v->c[c][p] = 0;
                    break;
                case LCS_SLIP: case LCS_INFLOW: case LCS_OUTFLOW: case LCS_2D: {
                    if (inside) break;
                    long b = PX(d, clampi(i, 1, d->ni), clampi(j, 1, d->nj), clampi(k, 1, d->nk));
                    for (int c = 0; c < 3; c++) v->c[c][p] = v->c[c][b];
                    break;
                }
                default: latch("set_velocity_bc: unknown bcflag");
                }
            }
}

/* set_flowmap_bc, flowmap_m.f90:325-392 */
static void set_flowmap_bc(const sgrid_t *g, sr1_t *fm) {
    const dims_t *d = &g->d;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long p = PX(d, i, j, k);
                int f = g->bcflag[p];
                if (f == LCS_MASK || f == LCS_INFLOW || f == LCS_OUTFLOW)
                    for (int c = 0; c < 3; c++) fm->c[c][p] = 0;
            }
    for (int k = 0; k <= d->nk + 1; k++)
        for (int j = 0; j <= d->nj + 1; j++)
            for (int i = 0; i <= d->ni + 1; i++) {
                if (i >= 1 && j >= 1 && k >= 1 && i <= d->ni && j <= d->nj && k <= d->nk) continue;
                long p = PX(d, i, j, k);
                switch (g->bcflag[p]) {
                case LCS_INTERNAL: break;
                case LCS_WALL: case LCS_MASK: case LCS_INFLOW: case LCS_OUTFLOW:
                    for (int c = 0; c < 3; c++) fm->c[c][p] = 0;
                    break;
                case LCS_SLIP: case LCS_2D: {
                    long b = PX(d, clampi(i, 1, d->ni), clampi(j, 1, d->nj), clampi(k, 1, d->nk));
                    for (int c = 0; c < 3; c++) fm->c[c][p] = fm->c[c][b];
                    break;
                }
                default: latch("set_flowmap_bc: unknown bcflag");
                }
            }
}

static void pad_flowmap(const sgrid_t *g, sr1_t *fm) {
    /* exchange_sdata(scomm_max_r1, fm) + set_flowmap_bc (flowmap_m.f90:90-91) */
    exchange_self(g, fm->c, 3, 1, 0);
    set_flowmap_bc(g, fm);
}

/* ------------------------------------------------------------------------------------
 * Lagrangian particle sets (lp_m.f90).
 * ------------------------------------------------------------------------------------ */
static void lp_alloc(lp_t *lp, int np) {
    lp->np = np;
    for (int c = 0; c < 3; c++) {
        lp->xp[c] = zalloc(np); lp->up[c] = zalloc(np); lp->dx[c] = zalloc(np);
        lp->no[c] = (int *)calloc((size_t)np, sizeof(int));
        lp->no_scfd[c] = (int *)calloc((size_t)np, sizeof(int));
    }
    lp->flag = (int *)calloc((size_t)np, sizeof(int));
}

/* reset_lp, lp_m.f90:228-294 (init_lp :13-114 is the same with fresh storage) */
static void reset_lp(const sgrid_t *g, lp_t *lp, int zero_fm) {
    const dims_t *d = &g->d;
    int ip = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++, ip++) {
                long p = PX(d, i, j, k);
                for (int c = 0; c < 3; c++) {
                    lp->xp[c][ip] = g->grid.c[c][p];
                    lp->up[c][ip] = 0;
                    lp->dx[c][ip] = 0;
                }
                lp->no[0][ip] = i; lp->no[1][ip] = j; lp->no[2][ip] = k;
                /* educated guess, lp_m.f90:276-278: nint(real(i*ni)/real(ni)) == i */
                /* (the solver grid S.g; g is the set's own grid, the same one at resolution 0) */
                lp->no_scfd[0][ip] = clampi(fnint((real)((float)(i * S.g.d.ni) / (float)d->ni)), 1, S.g.d.ni);
                lp->no_scfd[1][ip] = clampi(fnint((real)((float)(j * S.g.d.nj) / (float)d->nj)), 1, S.g.d.nj);
                lp->no_scfd[2][ip] = clampi(fnint((real)((float)(k * S.g.d.nk) / (float)d->nk)), 1, S.g.d.nk);
                lp->flag[ip] = LP_UNKNOWN;
            }
    lp->recursive_tracking = 1;
    if (zero_fm)
        for (int c = 0; c < 3; c++) memset(lp->fm.c[c], 0, sizeof(real) * (size_t)d->ntot);
}

/* project_lp2plane, lp_m.f90:418-538, for a rectilinear grid (its plane normal is the
 * singleton axis).  Returns immediately on 3-D grids (:433). */
static void project_lp2plane(const sgrid_t *g, lp_t *lp, int *const *no) {
    const dims_t *d = &g->d;
    if (g->gn[0] > 1 && g->gn[1] > 1 && g->gn[2] > 1) return;
    int ax = g->gn[2] == 1 ? 2 : (g->gn[1] == 1 ? 1 : 0);
    /* the last matching block wins in the reference; it also forces no%ax = 1 for both node sets */
    for (int ip = 0; ip < lp->np; ip++) {
        lp->no[ax][ip] = 1;
        lp->no_scfd[ax][ip] = 1;
    }
#pragma omp parallel for schedule(static)
    for (int ip = 0; ip < lp->np; ip++) {
        int i = clampi(no[0][ip], 1, d->ni), j = clampi(no[1][ip], 1, d->nj), k = clampi(no[2][ip], 1, d->nk);
        long p = PX(d, i, j, k);
        /* normal = v1 x v2 from central differences of the grid around the node */
        real v1[3], v2[3], nrm[3];
        int ip1 = i + 1, im1 = i - 1, jp1 = j + 1, jm1 = j - 1, kp1 = k + 1, km1 = k - 1;
        for (int c = 0; c < 3; c++) {
            if (ax == 0) {
                v1[c] = g->grid.c[c][PX(d, i, jp1, k)] - g->grid.c[c][PX(d, i, jm1, k)];
                v2[c] = g->grid.c[c][PX(d, i, j, kp1)] - g->grid.c[c][PX(d, i, j, km1)];
            } else if (ax == 1) {
                v1[c] = g->grid.c[c][PX(d, ip1, j, k)] - g->grid.c[c][PX(d, im1, j, k)];
                v2[c] = g->grid.c[c][PX(d, i, j, kp1)] - g->grid.c[c][PX(d, i, j, km1)];
            } else {
                v1[c] = g->grid.c[c][PX(d, ip1, j, k)] - g->grid.c[c][PX(d, im1, j, k)];
                v2[c] = g->grid.c[c][PX(d, i, jp1, k)] - g->grid.c[c][PX(d, i, jm1, k)];
            }
        }
        nrm[0] = v1[1] * v2[2] - v1[2] * v2[1];
        nrm[1] = v1[2] * v2[0] - v1[0] * v2[2];
        nrm[2] = v1[0] * v2[1] - v1[1] * v2[0];
        real mag = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        for (int c = 0; c < 3; c++) nrm[c] = nrm[c] / mag;
        real dd[3];
        for (int c = 0; c < 3; c++) dd[c] = lp->xp[c][ip] - g->grid.c[c][p];
        real dist = dd[0] * nrm[0] + dd[1] * nrm[1] + dd[2] * nrm[2];
        if (dist < 0) {
            dist = -dist;
            for (int c = 0; c < 3; c++) nrm[c] = -nrm[c];
        }
        for (int c = 0; c < 3; c++) lp->xp[c][ip] = lp->xp[c][ip] - dist * nrm[c];
    }
}

/* set_lp_bc, lp_tracking_m.f90:185-277 */
static void set_lp_bc(const sgrid_t *g, lp_t *lp, int *const *no) {
    const dims_t *d = &g->d;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int ip = 0; ip < lp->np; ip++) {
        int i = clampi(no[0][ip], 1, d->ni), j = clampi(no[1][ip], 1, d->nj), k = clampi(no[2][ip], 1, d->nk);
        no[0][ip] = i; no[1][ip] = j; no[2][ip] = k;
        lp->flag[ip] = LP_IB;
        long p = PX(d, i, j, k);
        int f = g->bcflag[p];
        int interior = i > 1 && j > 1 && k > 1 && i < d->ni && j < d->nj && k < d->nk;
        switch (f) {
        case LCS_INTERNAL: case LCS_2D: break;
        case LCS_MASK: case LCS_SLIP: case LCS_WALL: {
            if (f != LCS_MASK && interior) break;
            /* dot_product accumulates left to right */
            real dist = (lp->xp[0][ip] - g->grid.c[0][p]) * g->bcnorm.c[0][p] + (lp->xp[1][ip] - g->grid.c[1][p]) * g->bcnorm.c[1][p] +
                   (lp->xp[2][ip] - g->grid.c[2][p]) * g->bcnorm.c[2][p];
            if (dist > 0)
                for (int c = 0; c < 3; c++) lp->xp[c][ip] = lp->xp[c][ip] - g->bcnorm.c[c][p] * dist;
            break;
        }
        case LCS_INFLOW: case LCS_OUTFLOW:
            if (interior) break;
            lp->flag[ip] = LP_STICK;
            for (int c = 0; c < 3; c++) lp->xp[c][ip] = g->grid.c[c][p];
            break;
        default: bad = 1;
        }
    }
    if (bad) latch("set_lp_bc: unknown bcflag");
}

/* ------------------------------------------------------------------------------------
 * Tensor-product B-spline interpolation, restated from the algorithms used by the
 * vendored bspline-fortran (src/bspline/bspline_sub_module.f90): knots dbknot :1737-1785,
 * collocation + banded LU without pivoting dbintk/dbnfac/dbnslv :1896-2259 (basis values
 * by the Cox-de Boor recurrence of dbspvn :2288-2370), three transposing passes x,y,z
 * (db3ink :451-533), and evaluation by de Boor's recurrence (dbvalu :2397-2533) after the
 * interval search of dintrv (:2558-2634) with db3val's range rules (:574-656).
 * Arrays here are 0-based; knot t[m] is the reference's t(m+1).
 * ------------------------------------------------------------------------------------ */
static void bsp_knots(const real *x, int n, int k, real *t) {
    real rnot = x[n - 1] + (real)0.1 * (x[n - 1] - x[n - 2]);
    for (int j = 0; j < k; j++) {
        t[j] = x[0];
        t[n + j] = rnot;
    }
    if (k % 2 == 1) {
        int off = (k - 1) / 2 - k;
        for (int j = k + 1; j <= n; j++) t[j - 1] = (real)0.5 * (x[off + j - 1] + x[off + j]);
    } else {
        int off = k / 2 - k;
        for (int j = k + 1; j <= n; j++) t[j - 1] = x[off + j - 1];
    }
}

/* values of the k B-splines of order k that are non-zero on [t(left), t(left+1)) at xv;
 * left is 1-based as in the reference. */
static void bsp_basis(const real *t, int k, int left, real xv, real *b) {
    real dr[8], dl[8];
    b[0] = 1;
    for (int j = 1; j < k; j++) {
        dr[j] = t[left + j - 1] - xv;      /* t(left+j) - x */
        dl[j] = xv - t[left - j];          /* x - t(left+1-j) */
        real prev = 0;
        for (int l = 1; l <= j; l++) {
            real vm = b[l - 1] / (dr[l] + dl[j + 1 - l]);
            b[l - 1] = vm * dr[l] + prev;
            prev = vm * dl[j + 1 - l];
        }
        b[j] = prev;
    }
}

typedef struct {
    int n, k;
    real *t;   /* n + k knots */
    real *w;   /* band LU, (2k-1) x n column-major, middle row k-1 (0-based) */
    int ok;
} bsp_axis_t;

static void bsp_axis_setup(bsp_axis_t *a, const real *x, int n, int k) {
    a->n = n; a->k = k;
    a->t = zalloc(n + k);
    int nr = 2 * k - 1;
    a->w = zalloc((long)nr * n);
    a->ok = 1;
    bsp_knots(x, n, k, a->t);
    int left = k;
    for (int i = 1; i <= n; i++) {
        real xi = x[i - 1];
        int lim = imin(i + k, n + 1);
        left = imax(left, i);
        if (xi < a->t[left - 1]) { a->ok = 0; return; }
        int found = 0;
        while (1) {
            if (xi < a->t[left]) { found = 1; break; }
            left = left + 1;
            if (left >= lim) break;
        }
        if (!found) {
            left = left - 1;
            if (xi > a->t[left]) { a->ok = 0; return; }
        }
        real b[8];
        bsp_basis(a->t, k, left, xi, b);
        for (int j = 1; j <= k; j++) {
            int col = left - k + j;                /* 1-based column */
            int row = k + i - col;                 /* 1-based band row */
            a->w[(row - 1) + (long)nr * (col - 1)] = b[j - 1];
        }
    }
    /* dbnfac with nbandl = nbandu = k-1 */
    int mid = k; /* 1-based */
    int nb = k - 1;
    for (int i = 1; i <= n - 1; i++) {
        real piv = a->w[(mid - 1) + (long)nr * (i - 1)];
        if (piv == 0) { a->ok = 0; return; }
        int jmax = imin(nb, n - i);
        for (int j = 1; j <= jmax; j++) a->w[(mid + j - 1) + (long)nr * (i - 1)] = a->w[(mid + j - 1) + (long)nr * (i - 1)] / piv;
        int kmax = imin(nb, n - i);
        for (int kk = 1; kk <= kmax; kk++) {
            int ipk = i + kk, midmk = mid - kk;
            real fac = a->w[(midmk - 1) + (long)nr * (ipk - 1)];
            for (int j = 1; j <= jmax; j++)
                a->w[(midmk + j - 1) + (long)nr * (ipk - 1)] =
                    a->w[(midmk + j - 1) + (long)nr * (ipk - 1)] - a->w[(mid + j - 1) + (long)nr * (i - 1)] * fac;
        }
    }
    if (a->w[(mid - 1) + (long)nr * (n - 1)] == 0) a->ok = 0;
}

static void bsp_axis_free(bsp_axis_t *a) {
    free(a->t); free(a->w);
    a->t = a->w = NULL;
}

/* dbnslv: solve in place, b strided by `st` */
static void bsp_axis_solve(const bsp_axis_t *a, real *b, long st) {
    int n = a->n, k = a->k, nr = 2 * k - 1, mid = k, nb = k - 1;
    const real *w = a->w;
#define B(i) b[(long)((i)-1) * st]
#define W(r, c) w[((r)-1) + (long)nr * ((c)-1)]
    if (n != 1) {
        for (int i = 1; i <= n - 1; i++) {
            int jmax = imin(nb, n - i);
            for (int j = 1; j <= jmax; j++) B(i + j) = B(i + j) - B(i) * W(mid + j, i);
        }
        int i = n;
        while (1) {
            B(i) = B(i) / W(mid, i);
            int jmax = imin(nb, i - 1);
            for (int j = 1; j <= jmax; j++) B(i - j) = B(i - j) - B(i) * W(mid - j, i);
            i = i - 1;
            if (i <= 1) break;
        }
    }
    B(1) = B(1) / W(mid, 1);
#undef B
#undef W
}

typedef struct {
    bsp_axis_t ax[3];
    long nx, ny, nz;
    real *coef; /* x fastest */
} bsp3_t;

static void bsp3_setup(bsp3_t *s, const real *xg, const real *yg, const real *zg, int nx, int ny, int nz, int kx, int ky, int kz) {
    s->nx = nx; s->ny = ny; s->nz = nz;
    bsp_axis_setup(&s->ax[0], xg, nx, kx);
    bsp_axis_setup(&s->ax[1], yg, ny, ky);
    bsp_axis_setup(&s->ax[2], zg, nz, kz);
    s->coef = zalloc((long)nx * ny * nz);
}

static void bsp3_free(bsp3_t *s) {
    for (int a = 0; a < 3; a++) bsp_axis_free(&s->ax[a]);
    free(s->coef);
    s->coef = NULL;
}

/* fit: db3ink with iflag = 0 (knots by dbknot).  Order of the three passes: x, y, z. */
static void bsp3_fit(bsp3_t *s, const real *f) {
    long nx = s->nx, ny = s->ny, nz = s->nz;
    memcpy(s->coef, f, sizeof(real) * (size_t)(nx * ny * nz));
    if (!s->ax[0].ok || !s->ax[1].ok || !s->ax[2].ok) {
        latch("bspline: singular collocation system");
        return;
    }
#pragma omp parallel for schedule(static)
    for (long l = 0; l < ny * nz; l++) bsp_axis_solve(&s->ax[0], s->coef + l * nx, 1);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nx * nz; l++) {
        long i = l % nx, kk = l / nx;
        bsp_axis_solve(&s->ax[1], s->coef + i + kk * nx * ny, nx);
    }
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nx * ny; l++) bsp_axis_solve(&s->ax[2], s->coef + l, nx * ny);
}

/* dintrv: largest ileft (1-based) with xt(ileft) <= x; mflag -1 below, 1 at/above the end */
static int bsp_intrv(const real *xt, int lxt, real x, int *mflag) {
    if (x < xt[0]) { *mflag = -1; return 1; }
    if (x >= xt[lxt - 1]) { *mflag = 1; return lxt; }
    int lo = 1, hi = lxt; /* xt(lo) <= x < xt(hi) */
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (x >= xt[mid - 1]) lo = mid; else hi = mid;
    }
    *mflag = 0;
    return lo;
}

/* dbvalu with ideriv = 0; t points at the knot vector (0-based), a at n coefficients with
 * stride st.  Returns 0 and *bad = 1 where the reference returns an error. */
static real bsp_value(const real *t, const real *a, long st, int n, int k, real x, int *bad) {
    int mflag;
    int i = bsp_intrv(t, n + 1, x, &mflag);
    if (x < t[k - 1]) { *bad = 1; return 0; }
    if (mflag != 0) {
        if (x > t[i - 1]) { *bad = 1; return 0; }
        while (1) {
            if (i == k) { *bad = 1; return 0; }
            i = i - 1;
            if (x != t[i - 1]) break;
        }
    }
    real c[8], tr[8], tl[8];
    for (int j = 1; j <= k; j++) c[j - 1] = a[(long)(i - k + j - 1) * st];
    for (int j = 1; j <= k; j++) {
        tr[j] = t[i + j - 1] - x;       /* t(i+j) - x */
        tl[j] = x - t[i + 1 - j - 1];   /* x - t(i+1-j) */
    }
    for (int j = 1; j <= k - 1; j++) {
        int kmj = k - j, ilo = kmj;
        for (int jj = 1; jj <= kmj; jj++) {
            c[jj - 1] = (c[jj] * tl[ilo] + c[jj - 1] * tr[jj]) / (tl[ilo] + tr[jj]);
            ilo = ilo - 1;
        }
    }
    return c[0];
}

/* db3val: 0 outside [t(1), t(n+k)], 0 on any interval-search failure */
static real bsp3_eval(const bsp3_t *s, real x, real y, real z) {
    const bsp_axis_t *X = &s->ax[0], *Y = &s->ax[1], *Z = &s->ax[2];
    if (x < X->t[0] || x > X->t[X->n + X->k - 1]) return 0;
    if (y < Y->t[0] || y > Y->t[Y->n + Y->k - 1]) return 0;
    if (z < Z->t[0] || z > Z->t[Z->n + Z->k - 1]) return 0;
    int mf;
    int ly = bsp_intrv(Y->t, Y->n + Y->k, y, &mf);
    if (mf != 0) return 0;
    int lz = bsp_intrv(Z->t, Z->n + Z->k, z, &mf);
    if (mf != 0) return 0;
    real t1[8][8], t2[8];
    int bad = 0;
    long nx = s->nx, nxy = s->nx * s->ny;
    for (int kk = 1; kk <= Z->k; kk++) {
        int cz = lz - Z->k + kk;
        for (int jj = 1; jj <= Y->k; jj++) {
            int cy = ly - Y->k + jj;
            t1[kk - 1][jj - 1] = bsp_value(X->t, s->coef + (long)(cy - 1) * nx + (long)(cz - 1) * nxy, 1, X->n, X->k, x, &bad);
            if (bad) return 0;
        }
    }
    int ky0 = ly - Y->k + 1;
    for (int kk = 1; kk <= Z->k; kk++) {
        t2[kk - 1] = bsp_value(Y->t + (ky0 - 1), t1[kk - 1], 1, Y->k, Y->k, y, &bad);
        if (bad) return 0;
    }
    int kz0 = lz - Z->k + 1;
    return bsp_value(Z->t + (kz0 - 1), t2, 1, Z->k, Z->k, z, &bad);
}

/* ------------------------------------------------------------------------------------
 * interp_s2u_r1, lp_tracking_m.f90:279-662 (NEAREST_NBR, LINEAR, QUADRATIC, CUBIC, and
 * TSE / TSE_LIMIT with grad_sr1's central differences, gradient_m.f90:11-66; the
 * least-squares gradients of non-rectilinear grids are not restated: such grids are
 * rejected at init).
 * ------------------------------------------------------------------------------------ */
static void coord_lines(const sgrid_t *g, real **xg, real **yg, real **zg) {
    const dims_t *d = &g->d;
    *xg = zalloc(d->ni + 2); *yg = zalloc(d->nj + 2); *zg = zalloc(d->nk + 2);
    for (int i = 0; i <= d->ni + 1; i++) (*xg)[i] = g->grid.c[0][PX(d, i, 1, 1)];
    for (int j = 0; j <= d->nj + 1; j++) (*yg)[j] = g->grid.c[1][PX(d, 1, j, 1)];
    for (int k = 0; k <= d->nk + 1; k++) (*zg)[k] = g->grid.c[2][PX(d, 1, 1, k)];
    /* 2-D: fake unit spacing, lp_tracking_m.f90:367-378 */
    if (g->gn[0] == 1) { (*xg)[0] = (*xg)[1] - (real)1.0; (*xg)[2] = (*xg)[1] + (real)1.0; }
    if (g->gn[1] == 1) { (*yg)[0] = (*yg)[1] - (real)1.0; (*yg)[2] = (*yg)[1] + (real)1.0; }
    if (g->gn[2] == 1) { (*zg)[0] = (*zg)[1] - (real)1.0; (*zg)[2] = (*zg)[1] + (real)1.0; }
}

static void interp_r1(const sgrid_t *g, int method, int np, real *const *xp, int *const *no, const sr1_t *f, real *const *out) {
    const dims_t *d = &g->d;
    /* non-rectilinear grids: TSE_LIMIT unless TSE was asked for (lp_tracking_m.f90:320-327) */
    if (!g->rectilinear && method != TSE) method = TSE_LIMIT;
    switch (method) {
    case NEAREST_NBR:
#pragma omp parallel for schedule(static)
        for (int ip = 0; ip < np; ip++) {
            long p = PX(d, no[0][ip], no[1][ip], no[2][ip]);
            for (int c = 0; c < 3; c++) out[c][ip] = f->c[c][p];
        }
        break;
    case LINEAR: {
        real *xg, *yg, *zg;
        coord_lines(g, &xg, &yg, &zg);
        const real *L[3] = {xg, yg, zg};
        int nmax[3] = {d->ni + 1, d->nj + 1, d->nk + 1};
#pragma omp parallel for schedule(static)
        for (int ip = 0; ip < np; ip++) {
            int i0[3], i1[3];
            real t[3], mt[3];
            for (int a = 0; a < 3; a++) {
                int n0 = no[a][ip];
                if (xp[a][ip] > L[a][n0]) { i0[a] = n0; i1[a] = n0 + 1; }
                else { i0[a] = n0 - 1; i1[a] = n0; }
                /* the reference leaves an out-of-range bracket undefined; keep it in the array */
                i0[a] = clampi(i0[a], 0, nmax[a]); i1[a] = clampi(i1[a], 0, nmax[a]);
                real x0 = L[a][i0[a]], x1 = L[a][i1[a]];
                t[a] = (xp[a][ip] - x0) / (x1 - x0);
                t[a] = rmax(rmin(t[a], (real)1.0), (real)0.0);
                mt[a] = (real)1.0 - t[a];
            }
            long p0 = PX(d, i0[0], i0[1], i0[2]), p1 = PX(d, i1[0], i0[1], i0[2]);
            long p2 = PX(d, i0[0], i1[1], i0[2]), p3 = PX(d, i1[0], i1[1], i0[2]);
            long p4 = PX(d, i0[0], i0[1], i1[2]), p5 = PX(d, i1[0], i0[1], i1[2]);
            long p6 = PX(d, i0[0], i1[1], i1[2]), p7 = PX(d, i1[0], i1[1], i1[2]);
            for (int c = 0; c < 3; c++) {
                const real *F = f->c[c];
                out[c][ip] = mt[0] * mt[1] * mt[2] * F[p0] + t[0] * mt[1] * mt[2] * F[p1] + mt[0] * t[1] * mt[2] * F[p2] +
                             t[0] * t[1] * mt[2] * F[p3] + mt[0] * mt[1] * t[2] * F[p4] + t[0] * mt[1] * t[2] * F[p5] +
                             mt[0] * t[1] * t[2] * F[p6] + t[0] * t[1] * t[2] * F[p7];
            }
        }
        free(xg); free(yg); free(zg);
        break;
    }
    case QUADRATIC: case CUBIC: {
        int deg = method == QUADRATIC ? 2 : 3;
        real *xg, *yg, *zg;
        coord_lines(g, &xg, &yg, &zg);
        int nx = d->ni + 2, ny = d->nj + 2, nz = d->nk + 2;
        int kx = imax(imin(deg + 1, nx - 1), 2), ky = imax(imin(deg + 1, ny - 1), 2), kz = imax(imin(deg + 1, nz - 1), 2);
        bsp3_t s;
        bsp3_setup(&s, xg, yg, zg, nx, ny, nz, kx, ky, kz);
        for (int c = 0; c < 3; c++) {
            bsp3_fit(&s, f->c[c]);
#pragma omp parallel for schedule(static)
            for (int ip = 0; ip < np; ip++) out[c][ip] = bsp3_eval(&s, xp[0][ip], xp[1][ip], xp[2][ip]);
        }
        bsp3_free(&s);
        free(xg); free(yg); free(zg);
        break;
    }
    case TSE: case TSE_LIMIT: {
        /* lp_tracking_m.f90:526-654: phi(no) + grad(phi)(no) . (x - x(no)); grad_sr1 fills
         * interior nodes only (the ghost layer of the gradient array stays zero) and zeroes
         * the derivatives along a singleton axis; on non-rectilinear grids grad_sr1_ls
         * (face-neighbour least squares, zero on the ghost layer) replaces it.  TSE_LIMIT
         * clamps to the 27 values around no; at a ghost node the reference reads outside its
         * array there, and this restatement clips the window to the padded array. */
        const int lim = method == TSE_LIMIT;
        const int nn[3] = {d->ni, d->nj, d->nk};
        const long st[3] = {PX(d, 1, 0, 0) - PX(d, 0, 0, 0), PX(d, 0, 1, 0) - PX(d, 0, 0, 0), PX(d, 0, 0, 1) - PX(d, 0, 0, 0)};
#pragma omp parallel for schedule(static)
        for (int ip = 0; ip < np; ip++) {
            const int *q = (int[3]){no[0][ip], no[1][ip], no[2][ip]};
            long p = PX(d, q[0], q[1], q[2]);
            int interior = 1;
            for (int a = 0; a < 3; a++) interior &= q[a] >= 1 && q[a] <= nn[a];
            for (int c = 0; c < 3; c++) {
                const real *F = f->c[c];
                real gr[3] = {0, 0, 0}, dl[3];
                if (!g->rectilinear) grad_ls(g, F, q[0], q[1], q[2], gr);
                for (int a = 0; a < 3; a++) {
                    const real *X = g->grid.c[a];
                    if (g->rectilinear && interior && g->gn[a] != 1)
                        gr[a] = (F[p + st[a]] - F[p - st[a]]) / (X[p + st[a]] - X[p - st[a]]);
                    dl[a] = xp[a][ip] - X[p];
                }
                real r = F[p] + dl[0] * gr[0] + dl[1] * gr[1] + dl[2] * gr[2];
                if (lim) {
                    real mn = F[p], mx = F[p];
                    for (int k = imax(q[2] - 1, 0); k <= imin(q[2] + 1, d->nk + 1); k++)
                        for (int j = imax(q[1] - 1, 0); j <= imin(q[1] + 1, d->nj + 1); j++)
                            for (int i = imax(q[0] - 1, 0); i <= imin(q[0] + 1, d->ni + 1); i++) {
                                real v = F[PX(d, i, j, k)];
                                mn = rmin(mn, v);
                                mx = rmax(mx, v);
                            }
                    r = rmin(rmax(r, mn), mx);
                }
                out[c][ip] = r;
            }
        }
        break;
    }
    default:
        latch("interp: unsupported interpolator");
    }
}

/* ------------------------------------------------------------------------------------
 * Particle integration, lp_motion_m.f90:129-360
 * ------------------------------------------------------------------------------------ */
static real stage_ct(real tt, real t0, real t1) {
    /* ct = max(min((t-t0)/(t1-t0),1),0); the first update has t1 == t0 (0/0): the
     * displacement is 0 for any finite ct, so ct := 0 there. */
    if (t1 == t0) return 0;
    return rmax(rmin((tt - t0) / (t1 - t0), (real)1.0), (real)0.0);
}

static void blend(sr1_t *u, real ct) {
    const dims_t *d = &S.g.d;
    for (int c = 0; c < 3; c++) {
        real *U = u->c[c];
        const real *A = S.u_n.c[c], *B = S.u_np1.c[c];
#pragma omp parallel for schedule(static)
        for (long p = 0; p < d->ntot; p++) U[p] = ((real)1.0 - ct) * A[p] + ct * B[p];
    }
}

static void integrate_lp(lp_t *lp, real *t, real dt) {
    const sgrid_t *g = &S.g;
    int np = lp->np;
    const real HALF = (real)1.0 / (real)2.0, THIRD = (real)1.0 / (real)3.0, TWOTHIRD = (real)2.0 / (real)3.0,
               SIXTH = (real)1.0 / (real)6.0, TWO = (real)2.0;
    sr1_t u;
    sr1_alloc(&u, &g->d);
    real *xn[3], *k[3] = {0, 0, 0}, *xnp1[3] = {0, 0, 0};
    for (int c = 0; c < 3; c++) {
        xn[c] = zalloc(np);
        memcpy(xn[c], lp->xp[c], sizeof(real) * (size_t)np);
        if (S.integrator == RK3 || S.integrator == RK4) {
            k[c] = zalloc(np);
            xnp1[c] = zalloc(np);
        }
    }
    real t0 = S.t_n, t1 = S.t_np1, tt = *t;
    real **X = lp->xp, **U = lp->up;
    int *const *no = lp->no_scfd;
#define STAGE(ctv)                                   \
    do {                                             \
        blend(&u, (ctv));                            \
        interp_r1(g, S.interpolator, np, X, no, &u, U); \
    } while (0)
    switch (S.integrator) {
    case EULER:
        STAGE(stage_ct(tt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = X[c][ip] + dt * U[c][ip];
        break;
    case TRAPEZOIDAL:
        STAGE(stage_ct(tt + HALF * dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = X[c][ip] + dt * U[c][ip];
        break;
    case RK2:
        STAGE(stage_ct(tt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = X[c][ip] + HALF * dt * U[c][ip];
        STAGE(stage_ct(tt + HALF * dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = xn[c][ip] + dt * U[c][ip];
        break;
    case RK3:
        for (int c = 0; c < 3; c++) memcpy(xnp1[c], xn[c], sizeof(real) * (size_t)np);
        STAGE(stage_ct(tt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                xnp1[c][ip] = xnp1[c][ip] + SIXTH * k[c][ip];
            }
        /* stage 2 at xn + k1/2; the position set to xn - k1 at :239-241 is overwritten
         * before use, so stage 3 is evaluated at xn + 2*k2 (:245-247) */
        blend(&u, stage_ct(tt + HALF * dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = xn[c][ip] + HALF * k[c][ip];
        interp_r1(g, S.interpolator, np, X, no, &u, U);
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                X[c][ip] = xn[c][ip] + TWO * k[c][ip];
                xnp1[c][ip] = xnp1[c][ip] + TWOTHIRD * k[c][ip];
            }
        STAGE(stage_ct(tt + dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                X[c][ip] = xnp1[c][ip] + SIXTH * k[c][ip];
            }
        break;
    case RK4:
        for (int c = 0; c < 3; c++) memcpy(xnp1[c], xn[c], sizeof(real) * (size_t)np);
        STAGE(stage_ct(tt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                xnp1[c][ip] = xnp1[c][ip] + SIXTH * k[c][ip];
            }
        blend(&u, stage_ct(tt + HALF * dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = xn[c][ip] + HALF * k[c][ip];
        interp_r1(g, S.interpolator, np, X, no, &u, U);
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                xnp1[c][ip] = xnp1[c][ip] + THIRD * k[c][ip];
            }
        blend(&u, stage_ct(tt + HALF * dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = xn[c][ip] + HALF * k[c][ip];
        interp_r1(g, S.interpolator, np, X, no, &u, U);
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                xnp1[c][ip] = xnp1[c][ip] + THIRD * k[c][ip];
            }
        blend(&u, stage_ct(tt + dt, t0, t1));
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) X[c][ip] = xn[c][ip] + k[c][ip];
        interp_r1(g, S.interpolator, np, X, no, &u, U);
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                k[c][ip] = dt * U[c][ip];
                X[c][ip] = xnp1[c][ip] + SIXTH * k[c][ip];
            }
        break;
    default:
        latch("integrate_lp: unknown integrator");
    }
#undef STAGE
    *t = tt + dt;
    project_lp2plane(g, lp, lp->no_scfd);
    set_lp_bc(g, lp, lp->no_scfd);
    for (int ip = 0; ip < np; ip++)
        if (lp->flag[ip] == LP_STICK)
            for (int c = 0; c < 3; c++) X[c][ip] = xn[c][ip];
    for (int c = 0; c < 3; c++)
        for (int ip = 0; ip < np; ip++) lp->dx[c][ip] = lp->dx[c][ip] + (X[c][ip] - xn[c][ip]);
    for (int c = 0; c < 3; c++) {
        free(xn[c]); free(k[c]); free(xnp1[c]);
    }
    sr1_free(&u);
}

/* set_dt, lp_motion_m.f90:56-127 */
static int set_dt(const lp_t *lp, real *dt) {
    const dims_t *d = &S.g.d;
    real dt_f = S.t_np1 - S.t_n;
    real mx = -R_HUGE;
    int nan = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long p = PX(d, i, j, k);
                real c = 0;
                c = c + (real)fabs(S.u_np1.c[0][p] * S.delta.c[0][p]);
                c = c + (real)fabs(S.u_np1.c[1][p] * S.delta.c[1][p]);
                c = c + (real)fabs(S.u_np1.c[2][p] * S.delta.c[2][p]);
                c = c * dt_f;
                if (c != c) nan = 1;
                mx = rmax(mx, c);
            }
    if (nan) {
        latch("set_dt: non-finite velocity");
        return 1;
    }
    double q = ceil((double)(mx / (S.cfl_max * lp->dt_factor)));
    int nsub = (int)q;
    if (nsub < 1) nsub = 1;
    *dt = dt_f / (real)nsub;
    if (lp->direction == BKWD) *dt = (real)-1.0 * *dt;
    if (fabs(*dt) > 0) {
        if (lp->direction == FWD) S.integrations_fwd += (long long)lp->np * nsub;
        else S.integrations_bkwd += (long long)lp->np * nsub;
    }
    return nsub;
}

/* ------------------------------------------------------------------------------------
 * Node tracking with the one-rank periodic wrap of exchange_lpdata:
 * track_lp2node lp_tracking_m.f90:16-183, exchange_lpdata comms_m.f90:872-1189.
 * A recursive search repeats single passes until nothing moves (every particle is
 * independent, so "until this particle stops moving" is the same thing); the
 * reference gives up after 2*max(gn) passes (:127-142).
 * ------------------------------------------------------------------------------------ */
static int track_one_pass(const sgrid_t *g, const real *pos, int *node) {
    const dims_t *d = &g->d;
    real best = R_HUGE;
    int off[3] = {0, 0, 0};
    for (int nb = 0; nb < 27; nb++) {
        if (g->gn[0] == 1 && NBR[nb][0] != 0) continue;
        if (g->gn[1] == 1 && NBR[nb][1] != 0) continue;
        if (g->gn[2] == 1 && NBR[nb][2] != 0) continue;
        int i = clampi(node[0] + NBR[nb][0], 0, d->ni + 1);
        int j = clampi(node[1] + NBR[nb][1], 0, d->nj + 1);
        int k = clampi(node[2] + NBR[nb][2], 0, d->nk + 1);
        long p = PX(d, i, j, k);
        real ex = g->grid.c[0][p] - pos[0], ey = g->grid.c[1][p] - pos[1], ez = g->grid.c[2][p] - pos[2];
        real r = +ex * ex + ey * ey + ez * ez;
        if (r < (real)0.99 * best) {
            best = r;
            off[0] = NBR[nb][0]; off[1] = NBR[nb][1]; off[2] = NBR[nb][2];
        }
    }
    node[0] += off[0]; node[1] += off[1]; node[2] += off[2];
    return off[0] != 0 || off[1] != 0 || off[2] != 0;
}

static void wrap_lpdata(const sgrid_t *g, lp_t *lp, int ip, int *const *no) {
    const dims_t *d = &g->d;
    int n[3] = {d->ni, d->nj, d->nk};
    int cf[3];
    for (int a = 0; a < 3; a++) cf[a] = no[a][ip] < 1 ? -1 : (no[a][ip] > n[a] ? 1 : 0);
    if (cf[0] == 0 && cf[1] == 0 && cf[2] == 0) return;
    if (g->scomm_flag[cf[2] + 1][cf[1] + 1][cf[0] + 1] == NO_COMM) return;
    for (int a = 0; a < 3; a++) lp->xp[a][ip] = lp->xp[a][ip] + g->ps[cf[2] + 1][cf[1] + 1][cf[0] + 1][a];
    for (int a = 0; a < 3; a++) {
        int v = lp->no[a][ip];
        if (v > g->gn[a]) v -= g->gn[a];
        if (v < 1) v += g->gn[a];
        lp->no[a][ip] = v;
        v = lp->no_scfd[a][ip];
        if (v > g->gn[a]) v -= g->gn[a];
        if (v < 1) v += g->gn[a];
        lp->no_scfd[a][ip] = v;
    }
    lp->flag[ip] = LP_IB;
}

static void track_lp2node(const sgrid_t *g, lp_t *lp, int *const *no) {
    int recursive = lp->recursive_tracking;
    int maxtrack = 2 * imax(imax(g->gn[0], g->gn[1]), g->gn[2]);
    int fail = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : fail)
    for (int ip = 0; ip < lp->np; ip++) {
        int passes = 0;
        while (1) {
            real pos[3] = {lp->xp[0][ip], lp->xp[1][ip], lp->xp[2][ip]};
            int node[3] = {no[0][ip], no[1][ip], no[2][ip]};
            int moved = track_one_pass(g, pos, node);
            no[0][ip] = node[0]; no[1][ip] = node[1]; no[2][ip] = node[2];
            passes++;
            if (recursive && passes > maxtrack) { fail = 1; break; }
            if (lp->direction == FWD) wrap_lpdata(g, lp, ip, no);
            if (!recursive || !moved) break;
        }
    }
    if (fail) latch("track_lp2node: cannot locate all particles");
    lp->recursive_tracking = 0;
}

/* ------------------------------------------------------------------------------------
 * Backward SL flow-map update, flowmap_m.f90:17-104
 * ------------------------------------------------------------------------------------ */
static void update_flowmap_sl(lp_t *lp) {
    const sgrid_t *g = lp->sg;  /* the flow map's grid; the velocity is on S.g */
    const dims_t *d = &g->d;
    int np = lp->np;
    real dt;
    int nsub = set_dt(lp, &dt);
    if (S.error) return;
    S.last_nsub_bkwd = nsub;
    real *lpgrid[3], *fmp[3], *mask = zalloc(np);
    for (int c = 0; c < 3; c++) {
        lpgrid[c] = zalloc(np);
        fmp[c] = zalloc(np);
        memcpy(lpgrid[c], lp->xp[c], sizeof(real) * (size_t)np);
    }
    for (int ip = 0; ip < np; ip++)
        if (S.g.bcflag[PX(&S.g.d, lp->no_scfd[0][ip], lp->no_scfd[1][ip], lp->no_scfd[2][ip])] != LCS_MASK) mask[ip] = (real)1.0;
    real lp_time = S.t_np1;
    for (int sc = 1; sc <= nsub && !S.error; sc++) {
        integrate_lp(lp, &lp_time, dt);
        interp_r1(g, S.interpolator, np, lp->xp, lp->no, &lp->fm, fmp);
        for (int ip = 0; ip < np; ip++) {
            long p = PX(d, lp->no[0][ip], lp->no[1][ip], lp->no[2][ip]);
            for (int c = 0; c < 3; c++) lp->fm.c[c][p] = (fmp[c][ip] + (lp->xp[c][ip] - lpgrid[c][ip])) * mask[ip];
        }
        pad_flowmap(g, &lp->fm);
        for (int c = 0; c < 3; c++) memcpy(lp->xp[c], lpgrid[c], sizeof(real) * (size_t)np);
    }
    for (int c = 0; c < 3; c++) { free(lpgrid[c]); free(fmp[c]); }
    free(mask);
}

/* exchange_lpmap at one rank (comms_m.f90:1191-1376): fm(no0) = dx, particle order = node order */
static void lpmap_to_fm(lcs_t *L) {
    const dims_t *dl = &L->sg->d;
    int ip = 0;
    for (int k = 1; k <= dl->nk; k++)
        for (int j = 1; j <= dl->nj; j++)
            for (int ii = 1; ii <= dl->ni; ii++, ip++)
                for (int c = 0; c < 3; c++) L->lp.fm.c[c][PX(dl, ii, j, k)] = L->lp.dx[c][ip];
}

/* Forward particle update, lp_motion_m.f90:15-54 */
static void update_lp(lp_t *lp) {
    real dt;
    int nsub = set_dt(lp, &dt);
    if (S.error) return;
    S.last_nsub_fwd = nsub;
    real lp_time = S.t_n;
    for (int sc = 1; sc <= nsub && !S.error; sc++) {
        integrate_lp(lp, &lp_time, dt);
        lp->lifetime = lp->lifetime + (real)fabs((double)dt);
        track_lp2node(&S.g, lp, lp->no_scfd);
    }
}

/* ------------------------------------------------------------------------------------
 * Sub-flow-map ring and composition: write_flowmap_substep flowmap_m.f90:106-156,
 * reconstruct_flowmap :158-323, exchange_lp_alltoall comms_m.f90:1378-1709,
 * exchange_lpmap comms_m.f90:1191-1376.
 * ------------------------------------------------------------------------------------ */
static int ring_step(real t, real T, real h) {
    real m = (real)fmod((double)t, (double)T);
    return fnint(m / h);
}

static void write_substep(lcs_t *L) {
    const dims_t *d = &S.g.d;
    const dims_t *dl = &L->sg->d;
    int step = ring_step(S.t_np1, L->T, L->h);
    /* velocity snapshot (VELOCITY_INVARIANTS; step nint(T/h) is kept too: the forward
     * reconstruction reads step+1 before wrapping it) */
    if ((S.velocity_invariants || (S.write_lcs && !S.no_velocity_io)) && step >= 0 && step < MAXVSTEP) {
        long nint_ = (long)d->ni * d->nj * d->nk;
        for (int c = 0; c < 3; c++) {
            if (!S.vring[c][step]) S.vring[c][step] = zalloc(nint_);
            real *v = S.vring[c][step];
            long q = 0;
            for (int k = 1; k <= d->nk; k++)
                for (int j = 1; j <= d->nj; j++)
                    for (int i = 1; i <= d->ni; i++) v[q++] = S.u_np1.c[c][PX(d, i, j, k)];
        }
        S.vwritten[step] = 1;
    }
    /* slot nint(T/h) (and negative slots) are written to files that reconstruct never
     * reads back (it wraps step into [0, nstep-1] before reading) */
    if (step < 0 || step >= L->nslot) return;
    for (int c = 0; c < 3; c++) {
        real *s = L->slot[c][step];
        long q = 0;
        for (int k = 1; k <= dl->nk; k++)
            for (int j = 1; j <= dl->nj; j++)
                for (int i = 1; i <= dl->ni; i++) s[q++] = L->lp.fm.c[c][PX(dl, i, j, k)];
    }
    L->written[step] = 1;
}

static void alltoall_wrap(const sgrid_t *g, lp_t *lp, int ip) {
    const dims_t *d = &g->d;
    real *x = &lp->xp[0][ip], *y = &lp->xp[1][ip], *z = &lp->xp[2][ip];
    const real *bb = g->bb;
    int inside = *x >= bb[0] && *x <= bb[3] && *y >= bb[1] && *y <= bb[4] && *z >= bb[2] && *z <= bb[5];
    if (!inside) {
        for (int kk = -1; kk <= 1 && !inside; kk++)
            for (int jj = -1; jj <= 1 && !inside; jj++)
                for (int ii = -1; ii <= 1 && !inside; ii++) {
                    const real *s = g->ps[kk + 1][jj + 1][ii + 1];
                    if (*x - s[0] >= bb[0] && *x - s[0] <= bb[3] && *y - s[1] >= bb[1] && *y - s[1] <= bb[4] && *z - s[2] >= bb[2] &&
                        *z - s[2] <= bb[5]) {
                        *x = *x - s[0]; *y = *y - s[1]; *z = *z - s[2];
                        inside = 1;
                    }
                }
    }
    lp->up[0][ip] = lp->up[1][ip] = lp->up[2][ip] = 0;
    real s = rmax(rmin((*x - bb[0]) / (bb[3] - bb[0]), (real)1.0), (real)0.0);
    real t = rmax(rmin((*y - bb[1]) / (bb[4] - bb[1]), (real)1.0), (real)0.0);
    real u = rmax(rmin((*z - bb[2]) / (bb[5] - bb[2]), (real)1.0), (real)0.0);
    if (g->rectilinear) {
        /* nint(real(ni)*s): real(ni) is a default (single precision) real */
        lp->no[0][ip] = clampi(fnint((real)((float)d->ni) * s), 1, d->ni);
        lp->no[1][ip] = clampi(fnint((real)((float)d->nj) * t), 1, d->nj);
        lp->no[2][ip] = clampi(fnint((real)((float)d->nk) * u), 1, d->nk);
    } else {
        /* comms_m.f90:1662-1673: the node index guessed from the index positions of the
         * coordinate extremes, nint(1/3 (imin_x + imin_y + imin_z)) + nint(1/3 (s (imax_x -
         * imin_x) + t (imax_y - imin_y) + u (imax_z - imin_z))) per direction */
        const real onethird = (real)1.0 / (real)3.0;
        const int nn[3] = {d->ni, d->nj, d->nk};
        for (int a = 0; a < 3; a++) {
            int v = fnint(onethird * (g->ijk_min[0][a] + g->ijk_min[1][a] + g->ijk_min[2][a])) +
                    fnint(onethird * (s * (g->ijk_max[0][a] - g->ijk_min[0][a]) + t * (g->ijk_max[1][a] - g->ijk_min[1][a]) +
                                      u * (g->ijk_max[2][a] - g->ijk_min[2][a])));
            lp->no[a][ip] = clampi(v, 1, nn[a]);
        }
    }
    lp->flag[ip] = LP_UNKNOWN;
}

static int reconstruct(lcs_t *L) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    lp_t *lp = &L->lp;
    int np = lp->np;
    reset_lp(g, lp, 1);
    int step = ring_step(S.t_np1, L->T, L->h);
    int nstep = fnint(L->T / L->h);
    int inc;
    if (lp->direction == FWD) {
        inc = 1;
        step = step + inc;
    } else {
        inc = -1;
    }
    int saved_dir = lp->direction;
    lp->direction = FWD;
    int success = 1;
    for (int i = 1; i <= nstep && !S.error; i++) {
        if (step >= nstep) step = 0;
        if (step < 0) step = nstep - 1;
        if (step >= L->nslot || !L->written[step]) {
            step = step + inc;
            success = 0;
            continue;
        }
        for (int c = 0; c < 3; c++) {
            const real *s = L->slot[c][step];
            long q = 0;
            for (int k = 1; k <= d->nk; k++)
                for (int j = 1; j <= d->nj; j++)
                    for (int ii = 1; ii <= d->ni; ii++) lp->fm.c[c][PX(d, ii, j, k)] = s[q++];
        }
        pad_flowmap(g, &lp->fm);
        project_lp2plane(g, lp, lp->no);
        set_lp_bc(g, lp, lp->no);
        interp_r1(g, S.interpolator, np, lp->xp, lp->no, &lp->fm, lp->up);
        for (int c = 0; c < 3; c++)
            for (int ip = 0; ip < np; ip++) {
                lp->xp[c][ip] = lp->xp[c][ip] + lp->up[c][ip];
                lp->dx[c][ip] = lp->dx[c][ip] + lp->up[c][ip];
            }
        for (int ip = 0; ip < np; ip++) alltoall_wrap(g, lp, ip);
        lp->recursive_tracking = 1;
        track_lp2node(g, lp, lp->no);
        step = step + inc;
    }
    /* exchange_lpmap: fm(no0) = dx; particle order equals origin order on one rank */
    {
        int ip = 0;
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int ii = 1; ii <= d->ni; ii++, ip++)
                    for (int c = 0; c < 3; c++) lp->fm.c[c][PX(d, ii, j, k)] = lp->dx[c][ip];
    }
    pad_flowmap(g, &lp->fm);
    lp->direction = saved_dir;
    return success;
}

/* ------------------------------------------------------------------------------------
 * FTLE: compute_ftle lcs_m.f90:66-193 with grad_sr1 gradient_m.f90:11-66.  The eigen
 * solve replaces LAPACK DSYEV/SSYEV by cyclic Jacobi in long double (largest eigenvalue).
 * ------------------------------------------------------------------------------------ */
static long double eig3_max(const long double A_in[3][3]) {
    long double a[3][3];
    memcpy(a, A_in, sizeof(a));
    for (int sweep = 0; sweep < 64; sweep++) {
        long double off = fabsl(a[0][1]) + fabsl(a[0][2]) + fabsl(a[1][2]);
        long double diag = fabsl(a[0][0]) + fabsl(a[1][1]) + fabsl(a[2][2]);
        if (off == 0 || off <= 1e-30L * diag) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0) continue;
                long double theta = (a[q][q] - a[p][p]) / (2 * a[p][q]);
                long double tt = (theta >= 0 ? 1 : -1) / (fabsl(theta) + sqrtl(theta * theta + 1));
                long double c = 1 / sqrtl(tt * tt + 1), s = tt * c;
                for (int r = 0; r < 3; r++) {
                    long double arp = a[r][p], arq = a[r][q];
                    a[r][p] = c * arp - s * arq;
                    a[r][q] = s * arp + c * arq;
                }
                for (int r = 0; r < 3; r++) {
                    long double apr = a[p][r], aqr = a[q][r];
                    a[p][r] = c * apr - s * aqr;
                    a[q][r] = s * apr + c * aqr;
                }
            }
    }
    long double m = a[0][0];
    if (a[1][1] > m) m = a[1][1];
    if (a[2][2] > m) m = a[2][2];
    return m;
}

static void compute_ftle(lcs_t *L) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    sr1_t *fm = &L->lp.fm;
    exchange_self(g, fm->c, 3, 0, 0); /* scomm_face_r1 */
    const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long p = PX(d, i, j, k);
                long pxp = PX(d, i + 1, j, k), pxm = PX(d, i - 1, j, k);
                long pyp = PX(d, i, j + 1, k), pym = PX(d, i, j - 1, k);
                long pzp = PX(d, i, j, k + 1), pzm = PX(d, i, j, k - 1);
                real G[3][3]; /* G[c][a] = d fm_c / d x_a */
                if (L->naux) {
                    /* AUX_GRID (lcs_m.f90:95-127): differences of the X1/X0, Y1/Y0, Z1/Z0 maps over
                     * the aux grids' separation, left 0 where that is not above SMALL */
                    const real SMALL = (real)100.0 * R_TINY;
                    for (int a = 0; a < 3; a++) {
                        const lcs_t *A0 = L->aux[a], *A1 = L->aux[a + 3];
                        const real den = A1->sg->grid.c[a][p] - A0->sg->grid.c[a][p];
                        for (int c = 0; c < 3; c++)
                            G[c][a] = (real)fabs((double)den) > SMALL ? (A1->lp.fm.c[c][p] - A0->lp.fm.c[c][p]) / den : (real)0;
                    }
                } else if (!g->rectilinear) {
                    /* grad_sr1_ls (lcs_m.f90:129-133) */
                    for (int c = 0; c < 3; c++) grad_ls(g, fm->c[c], i, j, k, G[c]);
                } else {
                    for (int c = 0; c < 3; c++) {
                        const real *F = fm->c[c];
                        G[c][0] = (F[pxp] - F[pxm]) / (X[pxp] - X[pxm]);
                        G[c][1] = (F[pyp] - F[pym]) / (Y[pyp] - Y[pym]);
                        G[c][2] = (F[pzp] - F[pzm]) / (Z[pzp] - Z[pzm]);
                    }
                    for (int a = 0; a < 3; a++)
                        if (g->gn[a] == 1)
                            for (int c = 0; c < 3; c++) G[c][a] = 0;
                }
                /* cg_ab = sum_c G[c][a]*G[c][b], lcs_m.f90:137-145 */
                real C[3][3];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) C[a][b] = G[0][a] * G[0][b] + G[1][a] * G[1][b] + G[2][a] * G[2][b];
                long double A[3][3];
                /* DSYEV('V','U') reads the upper triangle */
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) A[a][b] = (long double)(a <= b ? C[a][b] : C[b][a]);
                real lam = (real)eig3_max(A);
                real sq = (real)sqrt((double)lam);
                /* max(sqrt(W3), tiny): a NaN from a rounding-negative W3 yields tiny */
                real mxv = (sq > R_TINY) ? sq : R_TINY;
                real v = (real)log((double)mxv) / L->T;
                if (S.incompressible) v = rmax(v, (real)0.0);
                L->ftle[p] = v;
            }
}

/* All three eigenvalues (ascending) of a symmetric 3x3, cyclic Jacobi in long double (the
 * DSYEV + sort3 of compute_invariants, invariants_m.f90:178-197, 210-237). */
static void eig3_all(const long double A_in[3][3], long double w[3]) {
    long double a[3][3];
    memcpy(a, A_in, sizeof(a));
    for (int sweep = 0; sweep < 64; sweep++) {
        long double off = fabsl(a[0][1]) + fabsl(a[0][2]) + fabsl(a[1][2]);
        long double diag = fabsl(a[0][0]) + fabsl(a[1][1]) + fabsl(a[2][2]);
        if (off == 0 || off <= 1e-30L * diag) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0) continue;
                long double theta = (a[q][q] - a[p][p]) / (2 * a[p][q]);
                long double tt = (theta >= 0 ? 1 : -1) / (fabsl(theta) + sqrtl(theta * theta + 1));
                long double c = 1 / sqrtl(tt * tt + 1), sn = tt * c;
                for (int r = 0; r < 3; r++) {
                    long double arp = a[r][p], arq = a[r][q];
                    a[r][p] = c * arp - sn * arq;
                    a[r][q] = sn * arp + c * arq;
                }
                for (int r = 0; r < 3; r++) {
                    long double apr = a[p][r], aqr = a[q][r];
                    a[p][r] = c * apr - sn * aqr;
                    a[q][r] = sn * apr + c * aqr;
                }
            }
    }
    long double x = a[0][0], y = a[1][1], z = a[2][2], t;
    if (y < x) { t = y; y = x; x = t; }
    if (z < y) { t = z; z = y; y = t; }
    if (y < x) { t = y; y = x; x = t; }
    w[0] = x; w[1] = y; w[2] = z;
}

/* compute_invariants, invariants_m.f90:15-208: the velocity at the frame's starting ring
 * step (reconstruct_flowmap reads it back and samples it at the grid nodes,
 * flowmap_m.f90:214-245 -- the nodal values, which LINEAR and NEAREST reproduce exactly and
 * the B-splines to rounding; a missing snapshot leaves the zeroed lp%ugrid), its central-
 * difference gradient with face exchange (grad_sr1, gradient_m.f90:11-66: periodic images,
 * zero ghosts elsewhere), and the Q, D, C, H and lambda-2 indicators. */
/* lp%ugrid of a frame (reconstruct_flowmap, flowmap_m.f90:214-245), on the set's own grid,
 * zero (reset_lp) unless the snapshot of ring step ustep exists.  On the solver grid: the nodal
 * values (the interpolators reproduce them at the nodes).  On a refined lcs grid: the
 * snapshot padded with its periodic images (other ghosts 0), interpolated with the global
 * interpolator at the lcs nodes around reset_lp's guessed solver nodes.  Periodic images of
 * the result (exchange_sdata, scomm_max_r1). */
static void make_ugrid(lcs_t *L, int ustep, sr1_t *ug) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    sr1_alloc(ug, d);
    if (!(ustep >= 0 && ustep < MAXVSTEP && S.vwritten[ustep])) return;
    if (g == &S.g) {
        for (int c = 0; c < 3; c++) {
            const real *v = S.vring[c][ustep];
            long q = 0;
            for (int k = 1; k <= d->nk; k++)
                for (int j = 1; j <= d->nj; j++)
                    for (int i = 1; i <= d->ni; i++) ug->c[c][PX(d, i, j, k)] = v[q++];
        }
    } else {
        const dims_t *ds = &S.g.d;
        sr1_t ut;
        sr1_alloc(&ut, ds);
        for (int c = 0; c < 3; c++) {
            const real *v = S.vring[c][ustep];
            long q = 0;
            for (int k = 1; k <= ds->nk; k++)
                for (int j = 1; j <= ds->nj; j++)
                    for (int i = 1; i <= ds->ni; i++) ut.c[c][PX(ds, i, j, k)] = v[q++];
        }
        exchange_self(&S.g, ut.c, 3, 1, 0);
        const int np = d->ni * d->nj * d->nk;
        real *xp[3], *up[3];
        int *no[3];
        for (int c = 0; c < 3; c++) {
            xp[c] = zalloc(np);
            up[c] = zalloc(np);
            no[c] = (int *)calloc((size_t)np, sizeof(int));
        }
        int ip = 0;
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++, ip++) {
                    for (int c = 0; c < 3; c++) xp[c][ip] = g->grid.c[c][PX(d, i, j, k)];
                    no[0][ip] = clampi(fnint((real)((float)(i * ds->ni) / (float)d->ni)), 1, ds->ni);
                    no[1][ip] = clampi(fnint((real)((float)(j * ds->nj) / (float)d->nj)), 1, ds->nj);
                    no[2][ip] = clampi(fnint((real)((float)(k * ds->nk) / (float)d->nk)), 1, ds->nk);
                }
        interp_r1(&S.g, S.interpolator, np, xp, no, &ut, up);
        ip = 0;
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++, ip++)
                    for (int c = 0; c < 3; c++) ug->c[c][PX(d, i, j, k)] = up[c][ip];
        for (int c = 0; c < 3; c++) { free(xp[c]); free(up[c]); free(no[c]); }
        sr1_free(&ut);
    }
    exchange_self(g, ug->c, 3, 1, 0); /* scomm_max_r1: periodic images, no boundary values */
}

static void compute_invariants(lcs_t *L, const sr1_t *ugp) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    const sr1_t ug = *ugp;
    const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
    const real eigth = (real)(1. / 8.), twenyforth = (real)(1. / 24.), coef = (real)(27. / 4.);
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long p = PX(d, i, j, k);
                long pxp = PX(d, i + 1, j, k), pxm = PX(d, i - 1, j, k);
                long pyp = PX(d, i, j + 1, k), pym = PX(d, i, j - 1, k);
                long pzp = PX(d, i, j, k + 1), pzm = PX(d, i, j, k - 1);
                real G[3][3]; /* G[c][a] = d u_c / d x_a */
                if (!g->rectilinear) {
                    /* grad_sr1_ls (invariants_m.f90:38-42) */
                    for (int c = 0; c < 3; c++) grad_ls(g, ug.c[c], i, j, k, G[c]);
                } else {
                    for (int c = 0; c < 3; c++) {
                        const real *F = ug.c[c];
                        G[c][0] = (F[pxp] - F[pxm]) / (X[pxp] - X[pxm]);
                        G[c][1] = (F[pyp] - F[pym]) / (Y[pyp] - Y[pym]);
                        G[c][2] = (F[pzp] - F[pzm]) / (Z[pzp] - Z[pzm]);
                    }
                    for (int a = 0; a < 3; a++)
                        if (g->gn[a] == 1)
                            for (int c = 0; c < 3; c++) G[c][a] = 0;
                }
                const real d1u1 = G[0][0], d2u1 = G[0][1], d3u1 = G[0][2];
                const real d1u2 = G[1][0], d2u2 = G[1][1], d3u2 = G[1][2];
                const real d1u3 = G[2][0], d2u3 = G[2][1], d3u3 = G[2][2];
                const real S11 = d1u1 + d1u1, S12 = d1u2 + d2u1, S13 = d1u3 + d3u1;
                const real S21 = d2u1 + d1u2, S22 = d2u2 + d2u2, S23 = d2u3 + d3u2;
                const real S31 = d3u1 + d1u3, S32 = d3u2 + d2u3, S33 = d3u3 + d3u3;
                const real W11 = d1u1 - d1u1, W12 = d1u2 - d2u1, W13 = d1u3 - d3u1;
                const real W21 = d2u1 - d1u2, W22 = d2u2 - d2u2, W23 = d2u3 - d3u2;
                const real W31 = d3u1 - d1u3, W32 = d3u2 - d2u3, W33 = d3u3 - d3u3;
                real INV[5];
                INV[0] = -eigth * (S11 * S11 + S12 * S21 + S13 * S31 + S21 * S12 + S22 * S22 + S23 * S32 + S31 * S13 + S32 * S23 +
                                   S33 * S33);
                INV[1] = -twenyforth *
                         (S11 * S11 * S11 + S11 * S12 * S21 + S11 * S13 * S31 + S21 * S11 * S12 + S21 * S12 * S22 + S21 * S13 * S32 +
                          S31 * S11 * S13 + S31 * S12 * S23 + S31 * S13 * S33 + S12 * S21 * S11 + S12 * S22 * S21 + S12 * S23 * S31 +
                          S13 * S31 * S11 + S13 * S32 * S21 + S13 * S33 * S31 + S22 * S22 * S22 + S22 * S21 * S12 + S22 * S23 * S32 +
                          S23 * S31 * S13 + S23 * S32 * S22 + S23 * S33 * S32 + S32 * S22 * S23 + S32 * S21 * S13 + S32 * S23 * S33 +
                          S33 * S33 * S33 + S33 * S23 * S32 + S33 * S13 * S31);
                INV[2] = INV[0] - eigth * (W11 * W11 + W12 * W21 + W13 * W31 + W21 * W12 + W22 * W22 + W23 * W32 + W31 * W13 +
                                           W32 * W23 + W33 * W33);
                INV[3] = INV[1] - eigth * (W11 * W11 * S11 + W11 * W12 * S21 + W11 * W13 * S31 + W21 * W11 * S12 + W21 * W12 * S22 +
                                           W21 * W13 * S32 + W31 * W11 * S13 + W31 * W12 * S23 + W31 * W13 * S33 + W12 * W21 * S11 +
                                           W12 * W22 * S21 + W12 * W23 * S31 + W13 * W31 * S11 + W13 * W32 * S21 + W13 * W33 * S31 +
                                           W22 * W22 * S22 + W22 * W21 * S12 + W22 * W23 * S32 + W23 * W31 * S13 + W23 * W32 * S22 +
                                           W23 * W33 * S32 + W32 * W22 * S23 + W32 * W21 * S13 + W32 * W23 * S33 + W33 * W33 * S33 +
                                           W33 * W23 * S32 + W33 * W13 * S31);
                INV[4] = INV[2] - INV[0];
                L->inv[0][p] = INV[2] > 0 ? (real)1 : (real)0;
                const real D = INV[2] * INV[2] * INV[2] + coef * INV[3] * INV[3];
                if (D > 0 && INV[3] > 0) L->inv[1][p] = 1;
                else if (D > 0 && INV[3] <= 0) L->inv[1][p] = 2;
                else if (D <= 0 && INV[3] > 0) L->inv[1][p] = 3;
                else L->inv[1][p] = 4;
                L->inv[2][p] = INV[1] > 0 ? (real)1 : (real)0;
                L->inv[3][p] = (real)sqrt((double)(-INV[4] / INV[0]));
                /* S^2 + Omega^2, upper triangle (DSYEV 'U') */
                long double A[3][3];
                A[0][0] = S11 * S11 + S21 * S12 + S31 * S13 + W11 * W11 + W21 * W12 + W31 * W13;
                A[0][1] = S12 * S11 + S22 * S12 + S32 * S13 + W12 * W11 + W22 * W12 + W32 * W13;
                A[0][2] = S13 * S11 + S23 * S12 + S33 * S13 + W13 * W11 + W23 * W12 + W33 * W13;
                A[1][1] = S12 * S21 + S22 * S22 + S32 * S23 + W12 * W21 + W22 * W22 + W32 * W23;
                A[1][2] = S13 * S21 + S23 * S22 + S33 * S23 + W13 * W21 + W23 * W22 + W33 * W23;
                A[2][2] = 0;
                A[1][0] = A[0][1];
                A[2][0] = A[0][2];
                A[2][1] = A[1][2];
                long double w[3];
                eig3_all(A, w);
                L->inv[4][p] = w[1] < 0 ? (real)1 : (real)0;
                long double big = fabsl(w[0]) > fabsl(w[2]) ? fabsl(w[0]) : fabsl(w[2]);
                L->l2margin[p] = big > 0 ? (real)(w[1] / big) : (real)0;
            }
}

/* Fortran ESw.d editing (the ES14.6 data and ES18.4 time fields of write_ftle): a signed
 * significand d.ddd... with one non-zero digit before the point (zero prints as 0.000...),
 * correctly rounded, then E+xx, or +xxx without the E for three-digit exponents; NaN and
 * Infinity as gfortran spells them; right-justified in w columns. */
static void es_edit(double v, int w, int d, char *out) {
    char b[64];
    int len;
    if (v != v) len = snprintf(b, sizeof b, "NaN");
    else if (v > DBL_MAX || v < -DBL_MAX) len = snprintf(b, sizeof b, "%s", v < 0 ? "-Infinity" : "Infinity");
    else {
        len = snprintf(b, sizeof b, "%.*E", d, v);
        char *e = strchr(b, 'E');
        if (e && (int)strlen(e + 2) == 3) { memmove(e, e + 1, strlen(e)); len--; }
    }
    if (len > w) { memset(out, '*', (size_t)w); return; }
    memset(out, ' ', (size_t)(w - len));
    memcpy(out + w - len, b, (size_t)len);
}

/* write_data_from_master (io_nohdf5_m.f90:266-332) at one rank: the interior of a padded
 * field (or a compact interior array when compact), i fastest, 10 values per line
 * (NDATA_PER_LINE; the MAX_CHUNK of 100000 is a multiple of 10, so chunking adds no breaks) */
static void write_block(FILE *fp, const dims_t *d, const real *f, int compact) {
    long count = (long)d->ni * d->nj * d->nk, q = 0;
    char cell[16];
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++, q++) {
                double v = f ? (double)(compact ? f[q] : f[PX(d, i, j, k)]) : 0.0;
                es_edit(v, 14, 6, cell);
                fwrite(cell, 1, 14, fp);
                if ((q + 1) % 10 == 0 || q + 1 == count) fputc('\n', fp);
            }
}

/* write_lcs + write_ftle (io_nohdf5_m.f90:47-133, 183-264): file name from the time index
 * (minus T/h for FTLE_FWD) with the reference's per-range integer formats, the Tecplot
 * header, then the X, Y, Z, [FM], [U], [FLAG], [Q C D H L2], FTLE blocks on the set's grid.
 * ug: lp%ugrid of the frame (make_ugrid). */
static void write_lcs(lcs_t *L, const sr1_t *ug) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    long long findex = (long long)fnint(S.t_np1 / L->h);
    if (L->diagnostic == FTLE_FWD) findex -= (long long)fnint(L->T / L->h);
    if (findex < -999999999LL || findex > 999999999LL) { latch("ERROR: unsupported range for file index"); return; }
    char idx[32];
    if (findex >= 1000 && findex <= 9999) snprintf(idx, sizeof idx, "%010lld", findex); /* i10.10 for this range */
    else snprintf(idx, sizeof idx, "%lld", findex);
    char path[1024];
    snprintf(path, sizeof path, "%s/%s_%s.dat", S.outdir[0] ? S.outdir : "./cfd2lcs_output", L->label, idx);
    FILE *fp = fopen(path, "w");
    if (!fp) { latch("write_lcs: cannot open the output file"); return; }
    fprintf(fp, "TITLE = \"%s-FTLE\"\nVARIABLES =\n\"X\"\n\"Y\"\n\"Z\"\n", L->label);
    if (!S.no_flowmap_io) fprintf(fp, "\"FM-X\"\n\"FM-Y\"\n\"FM-Z\"\n");
    if (!S.no_velocity_io) fprintf(fp, "\"U-X\"\n\"U-Y\"\n\"U-Z\"\n");
    if (S.bcflag_io) fprintf(fp, "\"FLAG\"\n");
    if (S.velocity_invariants) fprintf(fp, "\"Q\"\n\"C\"\n\"D\"\n\"H\"\n\"L2\"\n");
    char tfield[24];
    es_edit((double)S.t_np1, 18, 4, tfield);
    tfield[18] = 0;
    fprintf(fp, "\"FTLE\"\nZONE\nT = \"%s-FTLE\"\nSTRANDID = %010d, SOLUTIONTIME = %s\n", L->label, 1, tfield);
    fprintf(fp, "I = %010d J = %010d K = %010d\nZONETYPE = Ordered, DATAPACKING = BLOCK\n", d->ni, d->nj, d->nk);
    for (int c = 0; c < 3; c++) write_block(fp, d, g->grid.c[c], 0);
    if (!S.no_flowmap_io)
        for (int c = 0; c < 3; c++) write_block(fp, d, L->lp.fm.c[c], 0);
    if (!S.no_velocity_io)
        for (int c = 0; c < 3; c++) write_block(fp, d, ug->c[c], 0);
    if (S.bcflag_io) {
        long n = (long)d->ni * d->nj * d->nk, q = 0;
        real *fl = zalloc(n);
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++) fl[q++] = (real)g->bcflag[PX(d, i, j, k)];
        write_block(fp, d, fl, 1);
        free(fl);
    }
    if (S.velocity_invariants) {
        const int order[5] = {0, 2, 1, 3, 4}; /* Q, C, D, H, L2 */
        for (int q = 0; q < 5; q++) write_block(fp, d, L->inv[order[q]], 0);
    }
    write_block(fp, d, L->ftle, 0);
    fclose(fp);
}

/* write_tracers (io_nohdf5_m.f90:138-181) at one rank: POINT packing, x y z per particle;
 * STRANDID is lp%id + 1 (the particle set's number, here the diagnostic's). */
static void write_tracers(lcs_t *L) {
    long long findex = (long long)fnint(S.t_np1 / L->h);
    if (findex < -999999999LL || findex > 999999999LL) { latch("ERROR: unsupported range for file index"); return; }
    char idx[32];
    if (findex >= 1000 && findex <= 9999) snprintf(idx, sizeof idx, "%010lld", findex);
    else snprintf(idx, sizeof idx, "%lld", findex);
    char path[1024];
    snprintf(path, sizeof path, "%s/%s_%s.dat", S.outdir[0] ? S.outdir : "./cfd2lcs_output", L->label, idx);
    FILE *fp = fopen(path, "w");
    if (!fp) { latch("write_lcs: cannot open the output file"); return; }
    char tfield[24];
    es_edit((double)S.t_np1, 18, 4, tfield);
    tfield[18] = 0;
    fprintf(fp, "TITLE = \"%s-LP\"\nVARIABLES =\n\"X\"\n\"Y\"\n\"Z\"\nZONE\nT = \"%s-LP\"\n", L->label, L->label);
    fprintf(fp, "STRANDID = %010d, SOLUTIONTIME = %s\n", L->id + 1, tfield);
    fprintf(fp, "I = %010d J = %010d K = %010d\nZONETYPE = Ordered, DATAPACKING = POINT\n", L->lp.np, 1, 1);
    char cell[16];
    for (int ip = 0; ip < L->lp.np; ip++) {
        for (int c = 0; c < 3; c++) {
            es_edit((double)L->lp.xp[c][ip], 14, 6, cell);
            fwrite(cell, 1, 14, fp);
        }
        fputc('\n', fp);
    }
    fclose(fp);
}

/* ------------------------------------------------------------------------------------
 * Entry points (cfd2lcs.f90:2-682 semantics, one rank; output files only with WRITE_LCS).
 * ------------------------------------------------------------------------------------ */
#define EXPORT __attribute__((visibility("default")))

EXPORT int orc_real_size(void) { return (int)sizeof(real); }
EXPORT int orc_error(void) { return S.error; }
EXPORT const char *orc_error_msg(void) { return S.msg; }
EXPORT void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
EXPORT int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static void free_lcs(lcs_t *L) {
    if (!L) return;
    for (int m = 0; m < L->naux; m++) free_lcs(L->aux[m]);
    for (int c = 0; c < 3; c++) {
        free(L->lp.xp[c]); free(L->lp.up[c]); free(L->lp.dx[c]);
        free(L->lp.no[c]); free(L->lp.no_scfd[c]);
        if (L->slot[c]) {
            for (int s = 0; s < L->nslot; s++) free(L->slot[c][s]);
            free(L->slot[c]);
        }
    }
    free(L->lp.flag);
    for (int q = 0; q < 5; q++) free(L->inv[q]);
    free(L->l2margin);
    sr1_free(&L->lp.fm);
    sr1_free(&L->fm_out);
    free(L->ftle);
    free(L->written);
    if (L->own_sg) {
        sr1_free(&L->sg->grid); sr1_free(&L->sg->bcnorm); free(L->sg->bcflag);
        for (int nb = 0; nb < 6; nb++)
            for (int c = 0; c < 3; c++) free(L->sg->lsw[nb][c]);
        free(L->sg);
    }
    free(L);
}

/* Resets all state, including the error latch (a fresh process for the reference). */
EXPORT void orc_reset(void) {
    for (int i = 0; i < S.nlcs; i++) free_lcs(S.lcs[i]);
    for (int c = 0; c < 3; c++)
        for (int q = 0; q < MAXVSTEP; q++) free(S.vring[c][q]);
    if (S.inited) {
        sr1_free(&S.g.grid); sr1_free(&S.g.bcnorm); free(S.g.bcflag);
        for (int nb = 0; nb < 6; nb++)
            for (int c = 0; c < 3; c++) free(S.g.lsw[nb][c]);
        sr1_free(&S.u_n); sr1_free(&S.u_np1); sr1_free(&S.delta);
    }
    char keep[sizeof S.outdir];
    memcpy(keep, S.outdir, sizeof keep); /* the output directory outlives a reset */
    memset(&S, 0, sizeof(S));
    memcpy(S.outdir, keep, sizeof keep);
    S.integrator = RK2;
    S.interpolator = LINEAR;
    S.cfl_max = (real)0.5;
}

/* cfd2lcs_init, cfd2lcs.f90:2-53 */
EXPORT void orc_init(const int n[3], const int offset[3], const real *x, const real *y, const real *z, const int *flag) {
    (void)offset; /* one rank: offsets are normalised to 0 (sgrid_m.f90:90-93) */
    if (S.error) return;
    if (S.inited) orc_reset();
    S.nlcs = 0;
    S.integrations_fwd = S.integrations_bkwd = 0;
    if (init_sgrid(&S.g, n, x, y, z, flag)) return;
    sr1_alloc(&S.u_n, &S.g.d);
    sr1_alloc(&S.u_np1, &S.g.d);
    compute_delta(&S.g, &S.delta);
    S.first_call = 1;
    S.inited = 1;
}

/* cfd2lcs_diagnostic_init, cfd2lcs.f90:252-358 with init_ftle lcs_m.f90:16-64 */
/* directory of the output files (the reference's ./cfd2lcs_output) */
EXPORT void orc_set_output_dir(const char *dir) { snprintf(S.outdir, sizeof S.outdir, "%s", dir ? dir : ""); }

/* new_sgrid_from_sgrid (sgrid_m.f90:446-761) at one rank on a rectilinear grid.  res > 0:
 * res points between neighbouring nodes, x(ii) + dx * ir with dx = (x(ii+1) - x(ii)) / (res+1)
 * (the ghost image past the last node where the direction is periodic, nothing past it
 * otherwise); res < 0: every (|res|+1)-th node; singleton directions unchanged; each new point
 * inherits the flag of the node it starts from.  |res| >= n in a non-singleton direction
 * resets res to 0 (the reference's warning) and returns NULL, as res = 0 does. */
static sgrid_t *new_sgrid(int *res_io) {
    const sgrid_t *g = &S.g;
    const dims_t *d = &g->d;
    int res = *res_io;
    if (!g->rectilinear && res != 0) {
        latch("new_sgrid_from_sgrid: resolution /= 0 on a non-rectilinear grid is not restated");
        return NULL;
    }
    const int n[3] = {d->ni, d->nj, d->nk};
    for (int a = 0; a < 3; a++)
        if (n[a] > 1 && abs(res) >= n[a]) res = 0;
    *res_io = res;
    if (res == 0) return NULL;
    int nn[3];
    for (int a = 0; a < 3; a++) {
        if (n[a] == 1) { nn[a] = 1; continue; }
        nn[a] = 0;
        for (int i = 1; i <= n[a]; i++) {
            if (res > 0) {
                nn[a]++;
                for (int r = 1; r <= res; r++)
                    if (g->per[a] || i != n[a]) nn[a]++;
            } else if (i % (abs(res) + 1) == 0) {
                nn[a]++;
            }
        }
    }
    const long N = (long)nn[0] * nn[1] * nn[2];
    real *x = zalloc(N), *y = zalloc(N), *z = zalloc(N);
    int *fl = (int *)calloc((size_t)N, sizeof(int));
    const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
    if (res > 0) {
        for (int kk = 1; kk <= d->nk; kk++)
            for (int jj = 1; jj <= d->nj; jj++)
                for (int ii = 1; ii <= d->ni; ii++)
                    for (int kr = 0; kr <= res; kr++)
                        for (int jr = 0; jr <= res; jr++)
                            for (int ir = 0; ir <= res; ir++) {
                                const int in = ii + (ii - 1) * res + ir, jn = jj + (jj - 1) * res + jr, kn = kk + (kk - 1) * res + kr;
                                if (in > nn[0] || jn > nn[1] || kn > nn[2]) continue;
                                const long p = PX(d, ii, jj, kk);
                                const real dx0 = (X[PX(d, ii + 1, jj, kk)] - X[p]) / (real)(res + 1);
                                const real dx1 = (Y[PX(d, ii, jj + 1, kk)] - Y[p]) / (real)(res + 1);
                                const real dx2 = (Z[PX(d, ii, jj, kk + 1)] - Z[p]) / (real)(res + 1);
                                const long q = (in - 1) + (long)nn[0] * ((jn - 1) + (long)nn[1] * (kn - 1));
                                x[q] = X[p] + dx0 * (real)ir;
                                y[q] = Y[p] + dx1 * (real)jr;
                                z[q] = Z[p] + dx2 * (real)kr;
                                fl[q] = g->bcflag[p];
                            }
    } else {
        const int m = abs(res) + 1;
        int kn = 0;
        for (int k = 1; k <= d->nk; k++) {
            if (d->nk != 1 && k % m != 0) continue;
            kn++;
            int jn = 0;
            for (int j = 1; j <= d->nj; j++) {
                if (d->nj != 1 && j % m != 0) continue;
                jn++;
                int in = 0;
                for (int i = 1; i <= d->ni; i++) {
                    if (d->ni != 1 && i % m != 0) continue;
                    in++;
                    const long p = PX(d, i, j, k);
                    const long q = (in - 1) + (long)nn[0] * ((jn - 1) + (long)nn[1] * (kn - 1));
                    x[q] = X[p];
                    y[q] = Y[p];
                    z[q] = Z[p];
                    fl[q] = g->bcflag[p];
                }
            }
        }
    }
    sgrid_t *ng = (sgrid_t *)calloc(1, sizeof(sgrid_t));
    const int bad = init_sgrid(ng, nn, x, y, z, fl);
    free(x); free(y); free(z); free(fl);
    if (bad || !ng->rectilinear) {
        if (!S.error) latch("new_sgrid_from_sgrid: the new lcs grid is not rectilinear");
        free(ng);
        return NULL;
    }
    return ng;
}

/* LP_TRACER: init_lp_tracer (lp_m.f90:116-226) and diagnostic_init (cfd2lcs.f90:327-337):
 * one tracer per node with r <= TRACER_INJECT_RADIUS from the injection point, in node
 * order; none inside: the set is destroyed (its number used up) and the handle is -1. */
static int tracer_init(real T, real h, const char *label, int resolution) {
    /* lcs%sgrid: a refined copy when resolution /= 0 (its nodes are injected) */
    sgrid_t *sg = &S.g;
    int own = 0;
    if (resolution != 0) {
        sgrid_t *ng = new_sgrid(&resolution);
        if (S.error) return -1;
        if (ng) { sg = ng; own = 1; }
    }
    const dims_t *d = &sg->d;
    lcs_t *L = (lcs_t *)calloc(1, sizeof(lcs_t));
    L->id = S.nlcs + 1;
    L->diagnostic = LP_TRACER;
    L->sg = sg;
    L->own_sg = own;
    L->lp.sg = sg;
    L->T = T;
    L->h = h;
    snprintf(L->label, sizeof L->label, "%s", label ? label : "");
    for (size_t e = strlen(L->label); e > 0 && L->label[e - 1] == ' '; e--) L->label[e - 1] = 0;
    S.lcs[S.nlcs++] = L;
    real c0[3];
    for (int a = 0; a < 3; a++) c0[a] = S.tracer_set[a] ? S.tracer_c[a] : (real)R_HUGE;
    int np = 0;
    for (int pass = 0; pass < 2; pass++) {
        int ip = 0;
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++) {
                    long p = PX(d, i, j, k);
                    real dx = sg->grid.c[0][p] - c0[0], dy = sg->grid.c[1][p] - c0[1], dz = sg->grid.c[2][p] - c0[2];
                    real r = (real)sqrt((double)(dx * dx + dy * dy + dz * dz));
                    if (!(r <= S.tracer_r)) continue;
                    if (pass == 1) {
                        for (int c = 0; c < 3; c++) L->lp.xp[c][ip] = sg->grid.c[c][p];
                        L->lp.no[0][ip] = i; L->lp.no[1][ip] = j; L->lp.no[2][ip] = k;
                        /* init_lp_tracer's educated guess of the solver node */
                        L->lp.no_scfd[0][ip] = clampi(fnint((real)((float)(i * S.g.d.ni) / (float)d->ni)), 1, S.g.d.ni);
                        L->lp.no_scfd[1][ip] = clampi(fnint((real)((float)(j * S.g.d.nj) / (float)d->nj)), 1, S.g.d.nj);
                        L->lp.no_scfd[2][ip] = clampi(fnint((real)((float)(k * S.g.d.nk) / (float)d->nk)), 1, S.g.d.nk);
                        L->lp.flag[ip] = LP_UNKNOWN;
                    }
                    ip++;
                }
        if (pass == 0) {
            np = ip;
            if (np == 0) { L->dead = 1; return -1; }
            lp_alloc(&L->lp, np);
            sr1_alloc(&L->lp.fm, d);
        }
    }
    L->lp.direction = FWD;
    L->lp.dt_factor = (real)1.0;
    L->lp.recursive_tracking = 1;
    L->lp.lifetime = 0;
    track_lp2node(&S.g, &L->lp, L->lp.no_scfd);
    return L->id;
}

EXPORT int orc_tracer_count(int handle) {
    for (int i = 0; i < S.nlcs; i++)
        if (S.lcs[i]->id == handle) return S.lcs[i]->diagnostic == LP_TRACER ? S.lcs[i]->lp.np : -1;
    return -1;
}

EXPORT int orc_get_tracers(int handle, real *out) {
    for (int i = 0; i < S.nlcs; i++)
        if (S.lcs[i]->id == handle && S.lcs[i]->diagnostic == LP_TRACER) {
            const lp_t *lp = &S.lcs[i]->lp;
            for (int c = 0; c < 3; c++)
                for (int q = 0; q < lp->np; q++) out[(long)c * lp->np + q] = lp->xp[c][q];
            return 0;
        }
    return 1;
}

/* One auxiliary particle set on grid ag (init_lp on lcs%lpX0 ...): the parent's direction,
 * dt_factor, T and h, its own flow map and ring. */
static lcs_t *aux_set(const lcs_t *P, sgrid_t *ag) {
    const dims_t *d = &ag->d;
    lcs_t *A = (lcs_t *)calloc(1, sizeof(lcs_t));
    A->diagnostic = P->diagnostic;
    A->T = P->T;
    A->h = P->h;
    A->sg = ag;
    A->own_sg = 1;
    A->lp.sg = ag;
    lp_alloc(&A->lp, d->ni * d->nj * d->nk);
    sr1_alloc(&A->lp.fm, d);
    sr1_alloc(&A->fm_out, d);
    A->lp.direction = P->lp.direction;
    A->lp.dt_factor = P->lp.dt_factor;
    reset_lp(ag, &A->lp, 1);
    track_lp2node(&S.g, &A->lp, A->lp.no_scfd);
    A->nslot = P->nslot;
    A->written = (int *)calloc((size_t)A->nslot, sizeof(int));
    long nint_ = (long)d->ni * d->nj * d->nk;
    for (int c = 0; c < 3; c++) {
        A->slot[c] = (real **)calloc((size_t)A->nslot, sizeof(real *));
        for (int q = 0; q < A->nslot; q++) A->slot[c][q] = zalloc(nint_);
    }
    return A;
}

/* create_aux_grid (lcs_m.f90:225-435): per node, AUX_GRID_SCALING (0.2) times the mean
 * distance to its in-bounds face neighbours; six copies of the set's particles shifted by
 * -/+ that along x, y, z, projected into the data plane (2-D), each the nodes of a new grid
 * with the lcs grid's flags and a particle set of its own. */
static void create_aux(lcs_t *L) {
    const sgrid_t *g = L->sg;
    const dims_t *d = &g->d;
    const long N = (long)d->ni * d->nj * d->nk;
    const int n[3] = {d->ni, d->nj, d->nk};
    real *delta = zalloc(N);
    const real *X = g->grid.c[0], *Y = g->grid.c[1], *Z = g->grid.c[2];
    long q = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++, q++) {
                real nbrsum = 0, distsum = 0;
                for (int nb = 1; nb <= 6; nb++) {
                    const int ii = i + NBR[nb][0], jj = j + NBR[nb][1], kk = k + NBR[nb][2];
                    if (ii > 0 && jj > 0 && kk > 0 && ii <= d->ni && jj <= d->nj && kk <= d->nk) {
                        nbrsum = nbrsum + (real)1.0;
                        const long p = PX(d, i, j, k), pn = PX(d, ii, jj, kk);
                        const real dx = X[p] - X[pn], dy = Y[p] - Y[pn], dz = Z[p] - Z[pn];
                        distsum = distsum + (real)sqrt((double)(dx * dx + dy * dy + dz * dz));
                    }
                }
                delta[q] = distsum / nbrsum * (real)0.2;
            }
    real *xs[3] = {zalloc(N), zalloc(N), zalloc(N)};
    int *fl = (int *)calloc((size_t)N, sizeof(int));
    q = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) fl[q++] = g->bcflag[PX(d, i, j, k)];
    for (int m = 0; m < 6 && !S.error; m++) {
        const int a = m % 3;
        lp_t dum;
        memset(&dum, 0, sizeof dum);
        lp_alloc(&dum, (int)N);
        q = 0;
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++, q++) {
                    for (int c = 0; c < 3; c++) dum.xp[c][q] = L->lp.xp[c][q];
                    dum.xp[a][q] = m < 3 ? L->lp.xp[a][q] - delta[q] : L->lp.xp[a][q] + delta[q];
                    dum.no[0][q] = i; dum.no[1][q] = j; dum.no[2][q] = k;
                }
        project_lp2plane(g, &dum, dum.no);
        for (int c = 0; c < 3; c++) memcpy(xs[c], dum.xp[c], sizeof(real) * (size_t)N);
        for (int c = 0; c < 3; c++) { free(dum.xp[c]); free(dum.up[c]); free(dum.dx[c]); free(dum.no[c]); free(dum.no_scfd[c]); }
        free(dum.flag);
        sgrid_t *ag = (sgrid_t *)calloc(1, sizeof(sgrid_t));
        if (init_sgrid(ag, n, xs[0], xs[1], xs[2], fl) || !ag->rectilinear) {
            if (!S.error) latch("AUX_GRID: an auxiliary grid is not rectilinear (the TSE path is not restated)");
            free(ag);
            break;
        }
        L->aux[m] = aux_set(L, ag);
        L->naux = m + 1;
    }
    free(delta); free(fl);
    for (int c = 0; c < 3; c++) free(xs[c]);
}

EXPORT int orc_diagnostic_init(int type, int resolution, real T, real h, const char *label) {
    if (S.error) return -1;
    if (!S.inited) { latch("diagnostic_init before init"); return -1; }
    if (S.nlcs >= MAXLCS) { latch("diagnostic_init: too many diagnostics"); return -1; }
    if (type == LP_TRACER) return tracer_init(T, h, label, resolution);
    if (type != FTLE_FWD && type != FTLE_BKWD) {
        latch("ERROR, bad specification for lcs_type. Options are: FTLE_FWD, FTLE_BKWD, LP_TRACER");
        return -1;
    }
    /* lcs%sgrid: the solver grid, or new_sgrid_from_sgrid's copy (which may reset the
     * resolution to 0, changing dt_factor below as the reference's in-out argument does) */
    sgrid_t *sg = &S.g;
    int own = 0;
    if (resolution != 0) {
        sgrid_t *ng = new_sgrid(&resolution);
        if (S.error) return -1;
        if (ng) { sg = ng; own = 1; }
    }
    lcs_t *L = (lcs_t *)calloc(1, sizeof(lcs_t));
    L->id = S.nlcs + 1;
    L->diagnostic = type;
    L->T = T;
    L->h = h;
    L->sg = sg;
    L->own_sg = own;
    L->lp.sg = sg;
    snprintf(L->label, sizeof L->label, "%s", label ? label : "");
    for (size_t e = strlen(L->label); e > 0 && L->label[e - 1] == ' '; e--) L->label[e - 1] = 0; /* trim */
    const dims_t *d = &sg->d;
    L->ftle = zalloc(d->ntot);
    for (int q = 0; q < 5; q++) L->inv[q] = zalloc(d->ntot);
    L->l2margin = zalloc(d->ntot);
    lp_alloc(&L->lp, d->ni * d->nj * d->nk);
    sr1_alloc(&L->lp.fm, d);
    sr1_alloc(&L->fm_out, d);
    L->lp.direction = type == FTLE_BKWD ? BKWD : FWD;
    L->lp.dt_factor = type == FTLE_BKWD ? (real)1.0 / (real)imax(1 + resolution, 1) : (real)1.0;
    reset_lp(sg, &L->lp, 1);
    track_lp2node(&S.g, &L->lp, L->lp.no_scfd);
    L->nslot = fnint(T / h);
    if (L->nslot < 1) L->nslot = 1;
    L->written = (int *)calloc((size_t)L->nslot, sizeof(int));
    long nint_ = (long)d->ni * d->nj * d->nk;
    for (int c = 0; c < 3; c++) {
        L->slot[c] = (real **)calloc((size_t)L->nslot, sizeof(real *));
        for (int s = 0; s < L->nslot; s++) L->slot[c][s] = zalloc(nint_);
    }
    S.lcs[S.nlcs++] = L;
    if (S.aux_grid) {
        create_aux(L);
        if (S.error) return -1;
    }
    return L->id;
}

/* cfd2lcs_update, cfd2lcs.f90:55-250 */
EXPORT void orc_update(const int n[3], const real *u, const real *v, const real *w, real time) {
    if (S.error) return;
    if (!S.inited) { latch("update before init"); return; }
    const dims_t *d = &S.g.d;
    if (n[0] != d->ni || n[1] != d->nj || n[2] != d->nk) {
        latch("update: velocity array of incorrect dimension");
        return;
    }
    if (S.first_call) {
        S.t_n = time;
        S.t_np1 = time;
        S.first_call = 0;
    } else {
        S.t_n = S.t_np1;
        S.t_np1 = time;
    }
    for (int c = 0; c < 3; c++) memcpy(S.u_n.c[c], S.u_np1.c[c], sizeof(real) * (size_t)d->ntot);
    const real *src[3] = {u, v, w};
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) {
                long s = (i - 1) + (long)d->ni * ((j - 1) + (long)d->nj * (k - 1));
                for (int c = 0; c < 3; c++) S.u_np1.c[c][PX(d, i, j, k)] = src[c][s];
            }
    exchange_self(&S.g, S.u_np1.c, 3, 1, 0);
    set_velocity_bc(&S.g, &S.u_np1);
    for (int i = 0; i < S.nlcs && !S.error; i++) {
        if (S.lcs[i]->dead) continue;
        for (int m = -1; m < S.lcs[i]->naux && !S.error; m++) {
            lp_t *lp = m < 0 ? &S.lcs[i]->lp : &S.lcs[i]->aux[m]->lp;
            if (lp->direction == FWD) update_lp(lp);
            else update_flowmap_sl(lp);
        }
    }
    for (int i = 0; i < S.nlcs && !S.error; i++) {
        lcs_t *L = S.lcs[i];
        if (L->dead) continue;
        if ((long long)(S.t_np1 / L->h) == (long long)(S.t_n / L->h)) continue;
        if (L->diagnostic == LP_TRACER) { /* cfd2lcs.f90:225-231 */
            if (S.write_lcs) write_tracers(L);
            if (L->lp.lifetime > L->T) L->dead = 1;
            continue;
        }
        const dims_t *dl = &L->sg->d;
        if (L->diagnostic == FTLE_FWD) {
            /* exchange_lpmap: fm(no0) = dx */
            int ip = 0;
            for (int k = 1; k <= dl->nk; k++)
                for (int j = 1; j <= dl->nj; j++)
                    for (int ii = 1; ii <= dl->ni; ii++, ip++)
                        for (int c = 0; c < 3; c++) L->lp.fm.c[c][PX(dl, ii, j, k)] = L->lp.dx[c][ip];
        }
        if (S.aux_grid && !L->naux) {
            latch("AUX_GRID was set after cfd2lcs_diagnostic_init: no auxiliary particle sets exist");
            return;
        }
        /* the auxiliary sets go through the same substep, reconstruction and reset
         * (cfd2lcs.f90:151-222) */
        for (int m = 0; m < L->naux; m++) {
            if (L->diagnostic == FTLE_FWD) lpmap_to_fm(L->aux[m]);
            write_substep(L->aux[m]);
            reconstruct(L->aux[m]);
        }
        write_substep(L);
        /* the starting step of the reconstruction: the current one (backward) or the next,
         * not yet wrapped (forward), flowmap_m.f90:202-209 */
        const int ustep = ring_step(S.t_np1, L->T, L->h) + (L->diagnostic == FTLE_FWD ? 1 : 0);
        reconstruct(L);
        compute_ftle(L);
        sr1_t ug = {{NULL, NULL, NULL}};
        if (S.velocity_invariants || (S.write_lcs && !S.no_velocity_io)) make_ugrid(L, ustep, &ug);
        if (S.velocity_invariants) compute_invariants(L, &ug);
        if (S.write_lcs) write_lcs(L, &ug);
        sr1_free(&ug);
        for (int c = 0; c < 3; c++) memcpy(L->fm_out.c[c], L->lp.fm.c[c], sizeof(real) * (size_t)dl->ntot);
        S.ftle_frames++;
        reset_lp(L->sg, &L->lp, 1);
        track_lp2node(&S.g, &L->lp, L->lp.no_scfd);
        for (int m = 0; m < L->naux; m++) {
            reset_lp(L->aux[m]->sg, &L->aux[m]->lp, 1);
            track_lp2node(&S.g, &L->aux[m]->lp, L->aux[m]->lp.no_scfd);
        }
    }
}

/* cfd2lcs_set_option, cfd2lcs.f90:436-622 */
EXPORT void orc_set_option(const char *opt, int val) {
    if (S.error) return;
    int ok = 1;
    int tf = (val == LCS_TRUE || val == LCS_FALSE);
    if (!strcmp(opt, "SYNCTIMER") || !strcmp(opt, "DEBUG")) {
        ok = tf;
    } else if (!strcmp(opt, "WRITE_FLOWMAP")) {
        ok = tf;
        if (ok) S.no_flowmap_io = !val;
    } else if (!strcmp(opt, "WRITE_VELOCITY")) {
        ok = tf;
        if (ok) S.no_velocity_io = !val;
    } else if (!strcmp(opt, "WRITE_BCFLAG")) {
        ok = tf;
        if (ok) S.bcflag_io = val;
    } else if (!strcmp(opt, "WRITE_LCS")) { /* the library's switch for the output files */
        ok = tf;
        if (ok) S.write_lcs = val;
    } else if (!strcmp(opt, "VELOCITY_INVARIANTS")) {
        ok = tf;
        if (ok) S.velocity_invariants = val;
    } else if (!strcmp(opt, "INCOMPRESSIBLE")) {
        ok = tf;
        if (ok) S.incompressible = val;
    } else if (!strcmp(opt, "AUX_GRID")) {
        ok = tf;
        if (ok) S.aux_grid = val;
    } else if (!strcmp(opt, "UPDATE_FREQ")) {
        ok = 1;
    } else if (!strcmp(opt, "INTERPOLATOR")) {
        ok = val == NEAREST_NBR || val == LINEAR || val == QUADRATIC || val == CUBIC || val == TSE || val == TSE_LIMIT;
        S.interpolator = val; /* assigned even when the value is bad (cfd2lcs.f90:584) */
    } else if (!strcmp(opt, "INTEGRATOR")) {
        ok = val >= EULER && val <= RK4;
        S.integrator = val;
    } else {
        ok = 0;
    }
    if (!ok) latch("bad libcfd2lcs option/val combination");
}

/* cfd2lcs_set_param, cfd2lcs.f90:624-682 */
EXPORT void orc_set_param(const char *p, real val) {
    if (S.error) return;
    if (!strcmp(p, "CFL")) S.cfl_max = val;
    else if (!strcmp(p, "TRACER_INJECT_X")) { S.tracer_c[0] = val; S.tracer_set[0] = 1; }
    else if (!strcmp(p, "TRACER_INJECT_Y")) { S.tracer_c[1] = val; S.tracer_set[1] = 1; }
    else if (!strcmp(p, "TRACER_INJECT_Z")) { S.tracer_c[2] = val; S.tracer_set[2] = 1; }
    else if (!strcmp(p, "TRACER_INJECT_RADIUS")) S.tracer_r = val;
    else latch("unknown libcfd2lcs parameter");
}

static lcs_t *find_lcs(int handle) {
    for (int i = 0; i < S.nlcs; i++)
        if (S.lcs[i]->id == handle) return S.lcs[i];
    return NULL;
}

/* FTLE field of a diagnostic, interior points, i fastest */
EXPORT int orc_get_ftle(int handle, real *out) {
    lcs_t *L = find_lcs(handle);
    if (!L || !L->sg) return 1;
    const dims_t *d = &L->sg->d;
    long q = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) out[q++] = L->ftle[PX(d, i, j, k)];
    return 0;
}

/* Flow map (3 x interior, component-major) of a diagnostic: which = 0 the working
 * (sub-)flow map as currently stored, which = 1 the composed map of the last FTLE frame */
EXPORT int orc_get_fm(int handle, real *out, int which) {
    lcs_t *L = find_lcs(handle);
    if (!L || !L->sg) return 1;
    const dims_t *d = &L->sg->d;
    const sr1_t *f = which ? &L->fm_out : &L->lp.fm;
    long q = 0;
    for (int c = 0; c < 3; c++)
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++) out[q++] = f->c[c][PX(d, i, j, k)];
    return 0;
}

/* Grid points per direction of a diagnostic's lcs grid (the solver grid at resolution 0) */
EXPORT int orc_diag_size(int handle, int *n) {
    lcs_t *L = find_lcs(handle);
    if (!L || !L->sg) return 1;
    n[0] = L->sg->d.ni; n[1] = L->sg->d.nj; n[2] = L->sg->d.nk;
    return 0;
}

/* Forward particle positions (3 x np) of a diagnostic */
EXPORT int orc_get_particles(int handle, real *out) {
    lcs_t *L = find_lcs(handle);
    if (!L) return 1;
    long q = 0;
    for (int c = 0; c < 3; c++)
        for (int ip = 0; ip < L->lp.np; ip++) out[q++] = L->lp.xp[c][ip];
    return 0;
}

EXPORT long long orc_counter(int which) {
    switch (which) {
    case 0: return S.integrations_fwd;
    case 1: return S.integrations_bkwd;
    case 2: return S.last_nsub_fwd;
    case 3: return S.last_nsub_bkwd;
    case 4: return S.ftle_frames;
    default: return -1;
    }
}

/* Grid-derived quantities for host-logic tests: padded grid coordinates (3 x ntot),
 * padded bcflag (ntot), bcnorm (3 x ntot), inverse deltas (3 x ntot), periodicity. */
EXPORT long orc_padded_size(void) { return S.inited ? S.g.d.ntot : 0; }
EXPORT void orc_get_grid(real *xyz, int *flag, real *nrm, real *inv_delta, int *per) {
    const dims_t *d = &S.g.d;
    for (int c = 0; c < 3; c++) {
        if (xyz) memcpy(xyz + c * d->ntot, S.g.grid.c[c], sizeof(real) * (size_t)d->ntot);
        if (nrm) memcpy(nrm + c * d->ntot, S.g.bcnorm.c[c], sizeof(real) * (size_t)d->ntot);
        if (inv_delta) memcpy(inv_delta + c * d->ntot, S.delta.c[c], sizeof(real) * (size_t)d->ntot);
    }
    if (flag) memcpy(flag, S.g.bcflag, sizeof(int) * (size_t)d->ntot);
    if (per)
        for (int a = 0; a < 3; a++) per[a] = S.g.per[a];
}

/* Unit-level helpers (known-answer tests) */

/* interp_s2u_r1 with `method` on the initialised solver grid for np points (pts: x block, y
 * block, z block) with their nodes (padded indices, same layout); f3 holds three padded fields
 * of orc_padded_size() values, x fastest.  out receives the three components, one block each. */
/* compute_lsgw's face weights of a non-rectilinear grid: 18 padded arrays [nbr-2][component]
 * (all zero on a rectilinear grid); returns sgrid%rectilinear */
EXPORT int orc_get_lsq_weights(real *w) {
    const dims_t *d = &S.g.d;
    for (int nb = 0; nb < 6; nb++)
        for (int c = 0; c < 3; c++) {
            real *o = w + (long)(nb * 3 + c) * d->ntot;
            if (S.g.lsw[nb][c]) memcpy(o, S.g.lsw[nb][c], sizeof(real) * (size_t)d->ntot);
            else memset(o, 0, sizeof(real) * (size_t)d->ntot);
        }
    return S.g.rectilinear;
}

EXPORT int orc_interp_points(int method, const real *f3, int np, const real *pts, const int *nodes, real *out) {
    if (!S.inited) return 1;
    const long nt = S.g.d.ntot;
    sr1_t f;
    for (int c = 0; c < 3; c++) f.c[c] = (real *)f3 + c * nt;
    real *xp[3];
    int *no[3];
    real *o[3];
    for (int c = 0; c < 3; c++) {
        xp[c] = (real *)pts + (long)c * np;
        no[c] = (int *)nodes + (long)c * np;
        o[c] = out + (long)c * np;
    }
    interp_r1(&S.g, method, np, xp, no, &f, o);
    return S.error;
}
EXPORT double orc_eig3_max(const double *a9) {
    long double A[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[r][c] = (long double)a9[3 * r + c];
    return (double)eig3_max(A);
}

/* Fit a tensor spline of order (kx,ky,kz) to f (nx*ny*nz, x fastest) on lines xg,yg,zg and
 * evaluate it at npts points (px,py,pz). */
EXPORT int orc_bspline3(const real *xg, const real *yg, const real *zg, int nx, int ny, int nz, int kx, int ky, int kz, const real *f,
                        int npts, const real *px, const real *py, const real *pz, real *out) {
    bsp3_t s;
    bsp3_setup(&s, xg, yg, zg, nx, ny, nz, kx, ky, kz);
    if (!s.ax[0].ok || !s.ax[1].ok || !s.ax[2].ok) {
        bsp3_free(&s);
        return 1;
    }
    bsp3_fit(&s, f);
    for (int p = 0; p < npts; p++) out[p] = bsp3_eval(&s, px[p], py[p], pz[p]);
    bsp3_free(&s);
    return 0;
}

/* B-spline coefficients of the fit above (nx*ny*nz, x fastest) */
EXPORT int orc_bspline3_coef(const real *xg, const real *yg, const real *zg, int nx, int ny, int nz, int kx, int ky, int kz, const real *f,
                             real *coef) {
    bsp3_t s;
    bsp3_setup(&s, xg, yg, zg, nx, ny, nz, kx, ky, kz);
    if (!s.ax[0].ok || !s.ax[1].ok || !s.ax[2].ok) {
        bsp3_free(&s);
        return 1;
    }
    bsp3_fit(&s, f);
    memcpy(coef, s.coef, sizeof(real) * (size_t)(nx * ny * nz));
    bsp3_free(&s);
    return 0;
}

/* Velocity invariants of a diagnostic's last frame: 5 x interior (Q, D, C, H, L2). */
EXPORT int orc_get_invariants(int handle, real *out) {
    lcs_t *L = find_lcs(handle);
    if (!L || !L->sg) return 1;
    const dims_t *d = &L->sg->d;
    long q = 0;
    for (int v = 0; v < 5; v++)
        for (int k = 1; k <= d->nk; k++)
            for (int j = 1; j <= d->nj; j++)
                for (int i = 1; i <= d->ni; i++) out[q++] = L->inv[v][PX(d, i, j, k)];
    return 0;
}

/* Checker aid, no reference counterpart: the lambda-2 tie margin of the last frame, so that
 * a test can tell a rounding tie (|margin| at rounding level) from a real disagreement. */
EXPORT int orc_get_l2margin(int handle, real *out) {
    lcs_t *L = find_lcs(handle);
    if (!L || !L->sg) return 1;
    const dims_t *d = &L->sg->d;
    long q = 0;
    for (int k = 1; k <= d->nk; k++)
        for (int j = 1; j <= d->nj; j++)
            for (int i = 1; i <= d->ni; i++) out[q++] = L->l2margin[PX(d, i, j, k)];
    return 0;
}
