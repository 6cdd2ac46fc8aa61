// Host orchestration of libcfd2lcs_b200: owns the device state of one library instance
// (the reference keeps the same state in Fortran module globals, src/data_m.f90:313-387)
// and runs the per-update sequence of cfd2lcs_update (src/cfd2lcs.f90:55-250) as kernel
// launches on one CUDA stream.
#pragma once

#include <memory>
#include <string>
#include <vector>

#ifdef CFD2LCS_SP
typedef float lcsdata_t;
#else
typedef double lcsdata_t;
#endif

namespace cfd2lcs {

// User options (src/data_m.f90:19-92) plus the precision form of this library.
struct Options {
  int integrator = 2;     // RK2
  int interpolator = 1;   // LINEAR
  int incompressible = 0;
  int aux_grid = 0;
  int velocity_invariants = 0;
  double cfl = 0.5;
  int mixed_precision = 0;  // extension: FP32 velocity fields and interpolation taps, FP64 positions / flow maps
  // output files (write_lcs, src/io_nohdf5_m.f90:47-264): the variables written follow the
  // reference's FLOWMAP_IO, VELOCITY_IO and BCFLAG_IO defaults (src/data_m.f90:44-54)
  int write_flowmap = 1, write_velocity = 1, write_bcflag = 0;
  int write_lcs = 0;        // extension: write the files at all (off by default)
  // LP_TRACER injection sphere (cfd2lcs_set_param TRACER_INJECT_*, src/data_m.f90:86-89):
  // the default centre is huge(1.0), so no node is inside until the caller sets it
  double tracer_x = 1.0e300, tracer_y = 1.0e300, tracer_z = 1.0e300, tracer_r = 0.0;
  int write_lcs_async = 0;  // extension: let a frame's file complete after cfd2lcs_update returns
  // set for the batched form's instances: their kernels overlap other instances' on the device,
  // so their event times are not their own (the forward sets then re-sort on the fixed interval)
  int shared_device = 0;
};

struct Counters {
  long long integrations_fwd = 0, integrations_bkwd = 0;
  long long nsub_fwd = 0, nsub_bkwd = 0;
  long long ftle_frames = 0, updates = 0;
  long long kernel_launches = 0, slots_composed = 0;
  // event-timed hot kernels: backward SL subcycle and forward particle subcycle
  double sl_kernel_ms = 0, fwd_kernel_ms = 0;
  long long sl_kernel_launches = 0, fwd_kernel_launches = 0;
  // launches of the kernels that stage their spline taps in shared memory (backward, forward)
  long long sl_staged_launches = 0, fwd_staged_launches = 0;
  // of the staged backward launches, those of the LINEAR kernel that marches planes along z
  long long sl_march_launches = 0;
  // ingest, bkwd advect, fwd advect, snapshot, compose, ftle, whole update (event span)
  double phase_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

class EngineBase {
 public:
  virtual ~EngineBase() {}
  // false + msg on failure (the caller latches the error)
  virtual bool init(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag, std::string &msg) = 0;
  virtual int diagnostic_init(int type, int resolution, lcsdata_t T, lcsdata_t h, const char *label, std::string &msg) = 0;
  virtual bool update(const int n[3], const lcsdata_t *u, const lcsdata_t *v, const lcsdata_t *w, lcsdata_t time, bool device_ptrs,
                      std::string &msg) = 0;
  // update() in three parts: begin enqueues the ingest and the CFL read-back without waiting;
  // enqueue waits for that read-back only and enqueues the subcycles and the h-boundary work;
  // collect waits for the update's end and reads its timings and device error word
  virtual bool update_begin(const int n[3], const lcsdata_t *u, const lcsdata_t *v, const lcsdata_t *w, lcsdata_t time,
                            bool device_ptrs, std::string &msg) = 0;
  virtual bool update_enqueue(std::string &msg) = 0;
  virtual bool update_collect(std::string &msg) = 0;
  virtual bool get_ftle(int handle, lcsdata_t *out, std::string &msg) = 0;
  virtual bool get_flowmap(int handle, lcsdata_t *out, std::string &msg) = 0;
  virtual const lcsdata_t *ftle_device_ptr(int handle) = 0;
  // velocity invariants of the last frame (VELOCITY_INVARIANTS): 5 x interior (Q, D, C, H, L2)
  virtual bool get_invariants(int handle, lcsdata_t *out, std::string &msg) = 0;
  // LP_TRACER: particle count (-1 for another handle) and positions (x block, y, z)
  virtual int tracer_count(int handle) = 0;
  // points per direction of a diagnostic's lcs grid (the solver grid's unless resolution /= 0)
  virtual bool diagnostic_size(int handle, int n[3]) = 0;
  virtual bool get_tracers(int handle, lcsdata_t *out, std::string &msg) = 0;
  virtual bool sync_errors(std::string &msg) = 0;
  // Recomputes the latest FTLE frame of a diagnostic into caller-owned device buffers
  // without allocating (pointer table in a static device array, see engine.cu).
  virtual bool reconstruct_noalloc(int handle, lcsdata_t *d_ftle, lcsdata_t *d_fm, std::string &msg) = 0;
  // choices of the staged-versus-gathering tuner (family 0 backward, 1 forward) and the mean
  // launch times it measured per variant
  virtual void tuning(int choice[2], double ms[4]) const = 0;
  virtual const Counters &counters() const = 0;
  virtual bool host_grid_tables(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                                lcsdata_t *xyz_pad, int *flag_pad, lcsdata_t *nrm_pad, lcsdata_t *inv_delta, int *per,
                                std::string &msg) = 0;
};

// Creates the engine for the current options (plain precision of lcsdata_t, or mixed).
std::unique_ptr<EngineBase> make_engine(const Options *opt);

}  // namespace cfd2lcs
