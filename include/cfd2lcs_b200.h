/*
 * cfd2lcs_b200.h -- extensions of libcfd2lcs_b200 beyond the reference interface.
 * Include after cfd2lcs_inc_dp.h or cfd2lcs_inc_sp.h (lcsdata_t comes from there).
 *
 * The reference library has no return codes: an error latches a global flag and every
 * later call returns at once (src/cfd2lcs.f90:684-706).  These entry points keep that
 * convention and add ways to read the latch and the results (the reference only writes
 * them to files).
 */
#ifndef CFD2LCS_B200_H
#define CFD2LCS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Releases all host and device state (the reference's cfd2lcs_finalize,
 * src/cfd2lcs.f90:388-434, has no _c wrapper in src/cfd2lcs_c.c).  The error latch is
 * kept, as in the reference. */
void cfd2lcs_finalize_c(void);

/* Returns the error latch (0: no error) and copies the first error message into msg
 * (at most len bytes, NUL terminated).  Replaces reading CFD2LCS_ERROR, data_m.f90:380. */
int cfd2lcs_get_error_c(char *msg, size_t len);

/* Clears the error latch and all state, as a fresh process would start. */
void cfd2lcs_reset_c(void);

/* Copies the latest FTLE field of a diagnostic (n[0]*n[1]*n[2] values, i fastest) to host
 * memory.  The reference writes the same field to cfd2lcs_output/ (write_lcs,
 * src/io_nohdf5_m.f90:47-137).  Returns 0, or 1 for an unknown handle / no field yet. */
int cfd2lcs_get_ftle_c(int lcs_handle, lcsdata_t *ftle);

/* Copies the composed flow map (displacement form) of the latest FTLE frame: three
 * consecutive arrays (x, y, z components) of n[0]*n[1]*n[2] values each. */
int cfd2lcs_get_flowmap_c(int lcs_handle, lcsdata_t *fm);

/* cfd2lcs_update_c with u, v, w already resident in device memory (n[0]*n[1]*n[2] values
 * each, i fastest, same precision as lcsdata_t); no host copies. */
void cfd2lcs_update_device_c(int n[3], const lcsdata_t *d_u, const lcsdata_t *d_v, const lcsdata_t *d_w, lcsdata_t time);

/* Velocity invariants of a diagnostic's latest frame, computed when the option
 * VELOCITY_INVARIANTS is TRUE (compute_invariants, src/invariants_m.f90:15-208, which the
 * reference writes to its output file): five consecutive arrays of n[0]*n[1]*n[2] values (the
 * diagnostic's grid, cfd2lcs_diagnostic_size_c) --
 * Q-criterion flag, D zone (1..4), C (R_S > 0) flag, H and the lambda-2 flag.  Returns 0, or
 * 1 for an unknown handle, no frame yet or the option off. */
int cfd2lcs_get_invariants_c(int lcs_handle, lcsdata_t *inv);

/* Points per direction of a diagnostic's lcs grid.  With resolution /= 0 in
 * cfd2lcs_diagnostic_init (new_sgrid_from_sgrid, src/sgrid_m.f90:446-761) the FTLE field and
 * flow map live on a refined (res > 0: res points between neighbouring nodes) or coarsened
 * (res < 0: every (|res|+1)-th node) copy of the grid, and cfd2lcs_get_ftle_c /
 * cfd2lcs_get_flowmap_c return n[0]*n[1]*n[2] values of that grid.  0 on success. */
int cfd2lcs_diagnostic_size_c(int lcs_handle, int n[3]);

/* LP_TRACER diagnostics (cfd2lcs_diagnostic_init with LP_TRACER after setting the
 * TRACER_INJECT_X/Y/Z/RADIUS parameters; init_lp_tracer, src/lp_m.f90:116-226): one tracer per
 * grid node inside the injection sphere, advected forward every update until its lifetime
 * exceeds T.  The reference only writes their positions to its output files; these return
 * the count (-1 for a handle that is not a tracer set) and the positions, three consecutive
 * arrays (x, y, z) of count values each, the last ones reached.  0 on success. */
int cfd2lcs_tracer_count_c(int lcs_handle);
int cfd2lcs_get_tracers_c(int lcs_handle, lcsdata_t *xyz);

/* Device pointer of a diagnostic's latest FTLE field (n[0]*n[1]*n[2] doubles in the dp
 * build, floats in the sp build), valid until the next update or finalize. */
const lcsdata_t *cfd2lcs_ftle_device_ptr_c(int lcs_handle);

/* Work counters, as cfd2lcs_info prints them (src/cfd2lcs.f90:754-803):
 * counters[0] forward particle integrations (grid-pt x subcycles), cumulative
 * counters[1] backward particle integrations, cumulative
 * counters[2] subcycles of the last forward update, counters[3] of the last backward update
 * counters[4] FTLE frames computed, counters[5] updates
 * counters[6] kernel launches issued, counters[7] sub-flow maps composed */
void cfd2lcs_get_counters_c(long long counters[8]);

/* Device time (ms, CUDA events on the library's stream), cumulative:
 * t[0] ingest + padding (+ spline fit of the new velocity), t[1] backward advect,
 * t[2] forward advect, t[3] ring snapshot, t[4] composition, t[5] FTLE,
 * t[6] whole updates (first to last event of each update, host waits included). */
void cfd2lcs_get_phase_times_c(double t[7]);

/* Device time of the hot kernels alone (CUDA events around each launch), cumulative:
 * t[0] backward semi-Lagrangian subcycle kernels, t[1] forward particle kernels (ms);
 * n[0], n[1] the number of launches timed. */
void cfd2lcs_get_kernel_times_c(double t[2], long long n[2]);

/* Launches of the B-spline subcycle kernels that stage their coefficient taps in shared
 * memory (the cubic interpolator on 3-D grids), cumulative: n[0] backward semi-Lagrangian,
 * n[1] forward particle.  The rest of those launches gathered their taps from global memory. */
void cfd2lcs_get_staged_launches_c(long long n[2]);

/* Of the staged backward launches, those of the LINEAR kernel that marches planes of the
 * fields along z (FP64 grids whose rows are a multiple of 16 bytes), cumulative. */
void cfd2lcs_get_march_launches_c(long long *n);

/* The library times both forms of the cubic / LINEAR subcycle kernels -- taps staged in shared
 * memory or gathered from global memory, which give the same bits -- on an instance's first
 * launches and keeps the faster (environment CFD2LCS_B200_SL_TILE at cfd2lcs_init: 0 gathering
 * only, 1 tuned, the default, 2 staged wherever it applies).  choice[0] backward, choice[1]
 * forward kernel: -1 while sampling or where staging does not apply, 0 gathering, 1 staged;
 * ms[0], ms[1] the shortest backward launch times measured for gathering and staged (each
 * form's first launch left out), ms[2], ms[3] the forward ones. */
void cfd2lcs_get_tuning_c(int choice[2], double ms[4]);

/* Recomputes the latest FTLE frame of a diagnostic -- the composition of its stored
 * sub-flow maps and the FTLE -- into device buffers the caller owns, and allocates no memory
 * while doing so.  No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc at the point where they want the field, such as a CFD solver that hands the whole
 * GPU to its own memory pool at start-up and forbids allocations inside its time loop.
 *   d_ftle: n[0]*n[1]*n[2] values; d_fm: 3*n[0]*n[1]*n[2] values (x, y, z components), both
 *   device memory of lcsdata_t, i fastest.  The result equals cfd2lcs_get_ftle_c and
 *   cfd2lcs_get_flowmap_c of that frame when the options are unchanged since.
 * The table of sub-flow-map pointers lives in a fixed device array (256 sub-flow maps, i.e.
 * T/h <= 256; larger frames are rejected with an error).  The first call on a device looks
 * up that array's address.  The call copies the table from host memory and waits for its
 * own work, so it must not be made while a stream capture is active.  All calls share the
 * array, so calls that overlap on the GPU (from several host threads) race.
 * Ordering: the library writes d_ftle and d_fm on its own stream, which does not wait for
 * work the caller queued on other streams -- finish that work on both buffers before the
 * call.  The results are complete when the call returns.  The current CUDA device must be
 * the one cfd2lcs_init ran on.  Diagnostics with resolution /= 0 or AUX_GRID are rejected.
 * Returns 0 on success, 1 on error (the error is latched as for every other call). */
int cfd2lcs_reconstruct_noalloc_c(int lcs_handle, lcsdata_t *d_ftle, lcsdata_t *d_fm);

/* ---------------------------------------------------------------------------------------
 * Batched form.  No counterpart in the reference, which keeps one instance per process
 * (module globals, src/data_m.f90:313-387): here any number of independent instances -- each
 * with its own grid, options and diagnostics -- advance together.  A batch update starts the
 * velocity ingest of every listed instance on the instance's own stream, then enqueues every
 * instance's subcycles and FTLE frames, so the instances' kernels overlap on the GPU and the
 * host waits once per instance (for its CFL number).  The batch has its own error state and
 * leaves the reference-interface instance alone.  Functions return 0 (or an id >= 0) on
 * success and 1 (or -1) on error; cfd2lcs_batch_error_c gives the first error message.
 * ------------------------------------------------------------------------------------- */

/* Adds an instance on the grid (x, y, z, flag as for cfd2lcs_init_c) with its options
 * (integrator and interpolator codes of cfd2lcs_inc_*.h, CFL, MIXED_PRECISION 0/1).
 * Returns the instance id. */
int cfd2lcs_batch_add_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                        int integrator, int interpolator, lcsdata_t cfl, int mixed_precision);

/* cfd2lcs_diagnostic_init_c for one instance (resolution 0).  Returns the diagnostic handle
 * within that instance. */
int cfd2lcs_batch_diagnostic_init_c(int id, int lcs_type, lcsdata_t T, lcsdata_t h);

/* One update of `count` instances: ids[q] receives the device-resident velocity d_u[q],
 * d_v[q], d_w[q] (n[0]*n[1]*n[2] values of that instance, i fastest) at time[q]. */
int cfd2lcs_batch_update_device_c(int count, const int *ids, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                                  const lcsdata_t *const *d_w, const lcsdata_t *time);

/* Results and counters of one instance (as cfd2lcs_get_ftle_c, cfd2lcs_get_flowmap_c and
 * cfd2lcs_get_counters_c). */
int cfd2lcs_batch_get_ftle_c(int id, int lcs_handle, lcsdata_t *ftle);
int cfd2lcs_batch_get_flowmap_c(int id, int lcs_handle, lcsdata_t *fm);
int cfd2lcs_batch_get_counters_c(int id, long long counters[8]);

/* Number of instances; first error (0: none); release every instance and clear the error. */
int cfd2lcs_batch_size_c(void);
int cfd2lcs_batch_error_c(char *msg, size_t len);
void cfd2lcs_batch_reset_c(void);

/* ---------------------------------------------------------------------------------------
 * Adjoint.  No counterpart in the reference.  Gradient of J = sum_x weight(x) FTLE(x), the
 * backward FTLE of the whole horizon (the frame the library computes with h = T, T = time of
 * the last level minus the first), with respect to the velocity at every level, by a
 * hand-written reverse sweep through the semi-Lagrangian updates (LINEAR interpolation;
 * integrator EULER, TRAPEZOIDAL, RK2, RK3 or RK4) with a flow-map checkpoint every `checkpoint_every`
 * updates.  Grid: rectilinear, three-dimensional, every direction periodic, no boundary
 * flags.  d_u[l], d_v[l], d_w[l]: device arrays of level l (n[0]*n[1]*n[2], i fastest);
 * times: host, increasing; d_weight: device, n[0]*n[1]*n[2].  Writes *J and, when d_gu,
 * d_gv, d_gw are not NULL, dJ/du of every level into those device arrays.  Discrete choices
 * of the forward map (subcycle counts, interpolation brackets, clamped weights) are held
 * fixed.  Allocates device memory for the levels, their adjoints and the checkpoints.
 * Returns 0, or 1 with the reason in msg (at most len bytes). */
int cfd2lcs_adjoint_ftle_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, int integrator,
                           lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                           const lcsdata_t *const *d_w, const lcsdata_t *times, const lcsdata_t *d_weight, int checkpoint_every,
                           double *J, lcsdata_t *const *d_gu, lcsdata_t *const *d_gv, lcsdata_t *const *d_gw, char *msg, size_t len);

/* Tangent-linear model of the same objective (the forward-mode check of the adjoint): writes *J
 * and *dJ = sum over levels of <dJ/du, d> for one direction d (d_du[l], d_dv[l], d_dw[l]:
 * device arrays of level l, n[0]*n[1]*n[2], i fastest), propagating the flow map's first-order
 * change alongside the flow map with the same held-fixed discrete choices as the adjoint, so
 * that the two agree to rounding.  Same grid scope and arguments as cfd2lcs_adjoint_ftle_c.
 * Returns 0, or 1 with the reason in msg. */
int cfd2lcs_tangent_ftle_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, int integrator,
                           lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                           const lcsdata_t *const *d_w, const lcsdata_t *times, const lcsdata_t *d_weight,
                           const lcsdata_t *const *d_du, const lcsdata_t *const *d_dv, const lcsdata_t *const *d_dw, double *J,
                           double *dJ, char *msg, size_t len);

/* The two calls above with the boundary flags and the interpolator given.  flag: n[0]*n[1]*n[2]
 * values as cfd2lcs_init takes them, or NULL for all LCS_INTERNAL (the calls above); with LINEAR
 * interpolation any rectilinear grid, walled, with inflow / outflow, masked or 2-D, whose
 * particle boundary conditions and ghost rules the sweeps differentiate (projections along the
 * boundary normal and the plane, sticks and zeroed values held as the forward took them).
 * interpolator: LINEAR or CUBIC (the not-a-knot cubic B-spline of every axis, the library's cubic
 * path; three-dimensional periodic grids without flags, at least 3 points per direction).  With
 * CUBIC the reverse sweep scatters into the spline coefficients and carries that adjoint back
 * through the transposed banded solves of each fit; the tangent model fits the direction's
 * levels and the tangent map alongside. */
int cfd2lcs_adjoint_ftle_interp_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag, int integrator,
                                  int interpolator, lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u,
                                  const lcsdata_t *const *d_v, const lcsdata_t *const *d_w, const lcsdata_t *times,
                                  const lcsdata_t *d_weight, int checkpoint_every, double *J, lcsdata_t *const *d_gu,
                                  lcsdata_t *const *d_gv, lcsdata_t *const *d_gw, char *msg, size_t len);
int cfd2lcs_tangent_ftle_interp_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag, int integrator,
                                  int interpolator, lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u,
                                  const lcsdata_t *const *d_v, const lcsdata_t *const *d_w, const lcsdata_t *times,
                                  const lcsdata_t *d_weight, const lcsdata_t *const *d_du, const lcsdata_t *const *d_dv,
                                  const lcsdata_t *const *d_dw, double *J, double *dJ, char *msg, size_t len);


#ifdef __cplusplus
}
#endif

#endif
