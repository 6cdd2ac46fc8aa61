// C ABI of libcfd2lcs_b200: the reference's C entry points (src/cfd2lcs_c.c:67-142), the
// gfortran-mangled Fortran entry points (src/cfd2lcs.f90:2-682, external subroutines
// cfd2lcs_*_ with by-reference arguments and hidden character lengths), and the
// extensions declared in include/cfd2lcs_b200.h.
//
// Error convention as in the reference (src/cfd2lcs.f90:684-706): no return codes; the
// first error latches a flag, is reported once on stdout, and every later call returns
// immediately.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "adjoint.h"
#include "engine.h"
#include "grid.h"
#include "writer.h"

using cfd2lcs::Counters;
using cfd2lcs::EngineBase;
using cfd2lcs::HostGrid;
using cfd2lcs::Options;

#define CFD2LCS_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

enum { LCS_FALSE = 0, LCS_TRUE = 1 };
enum { NEAREST_NBR = 0, LINEAR = 1, QUADRATIC = 2, CUBIC = 3, TSE = 5, TSE_LIMIT = 6 };
enum { EULER = 0, TRAPEZOIDAL = 1, RK2 = 2, RK3 = 3, RK4 = 4 };

// State of the cfd2lcs_info table (cumulative times in seconds)
struct InfoState {
  bool started = false;
  std::chrono::steady_clock::time_point t_last;
  Counters prev;
  double total_sim = 0, total_lcs = 0, fwd = 0, bkwd = 0, reconstruct = 0, ftle = 0;
  long long fwd_n = 0, bkwd_n = 0;
  double fwd_s = 0, bkwd_s = 0;
};

struct Library {
  int error = 0;
  std::string msg;
  Options opt;
  std::unique_ptr<EngineBase> eng;
  bool inited = false;
  bool sync_timer = false;
  Counters zero;
  InfoState info;
};

Library &L() {
  static Library lib;
  return lib;
}

bool quiet() {
  const char *q = std::getenv("CFD2LCS_B200_QUIET");
  return q && q[0] && q[0] != '0';
}

void latch(const std::string &m) {
  Library &lib = L();
  if (!lib.error) {
    lib.msg = m;
    if (!quiet()) std::printf("ERROR (libcfd2lcs_b200): %s\nFATAL CFD2LCS_ERROR DETECTED, WILL NOT PERFORM LCS COMPUTATIONS\n", m.c_str());
  }
  lib.error = 1;
}

// Fortran character argument: trailing blanks are insignificant (trim()).  The reference's
// C shim passes the length as int while gfortran >= 8 reads size_t; only the low 32 bits
// are used and the string is also bounded by a NUL.
std::string fstr(const char *s, size_t len) {
  size_t n = (size_t)(uint32_t)len;
  n = strnlen(s, n);
  while (n > 0 && s[n - 1] == ' ') n--;
  return std::string(s, n);
}

void do_init(const int *n, const int *offset, const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag) {
  (void)offset;  // one rank: offsets are normalised to 0 (src/sgrid_m.f90:90-93)
  Library &lib = L();
  if (lib.error) return;
  lib.eng.reset();
  lib.inited = false;
  lib.info = InfoState();
  lib.eng = cfd2lcs::make_engine(&lib.opt);
  std::string msg;
  if (!lib.eng->init(n, x, y, z, flag, msg)) {
    lib.eng.reset();
    latch(msg);
    return;
  }
  lib.inited = true;
}

int do_diagnostic_init(int type, int resolution, lcsdata_t T, lcsdata_t h, const char *label) {
  Library &lib = L();
  if (lib.error) return -1;
  if (!lib.inited) {
    latch("cfd2lcs_diagnostic_init called before cfd2lcs_init");
    return -1;
  }
  std::string msg;
  const int id = lib.eng->diagnostic_init(type, resolution, T, h, label, msg);
  if (id == -2) return -1;  // LP_TRACER with no node in the injection sphere: handle -1, no error
  if (id < 0) latch(msg);
  return id;
}

// cfd2lcs_info (src/cfd2lcs.f90:708-810): the reference's table of time per phase and particle
// integration rates after every update, printed here when CFD2LCS_B200_INFO is set (off by
// default, so that a solver's standard output stays its own).  The first call only starts the
// clock, as in the reference.  Phase times are the device's (CUDA events): FWD / BKWD Advect,
// Reconstruct (snapshot + composition), LCS (FTLE); the I/O, LP re-map and error-check phases of
// the reference have no device counterpart here (0); "Other" is the rest of the update (ingest
// and the CFL read-back).  Application total is the wall clock from one update's end to the next.
void print_info() {
  Library &lib = L();
  const char *e = std::getenv("CFD2LCS_B200_INFO");
  if (lib.error || !lib.eng || !e || !e[0] || e[0] == '0') return;
  InfoState &I = lib.info;
  const auto now = std::chrono::steady_clock::now();
  const Counters &c = lib.eng->counters();
  if (!I.started) {
    I = InfoState();
    I.started = true;
    I.t_last = now;
    I.prev = c;
    return;
  }
  const Counters &p = I.prev;
  const double s_fwd = (c.phase_ms[2] - p.phase_ms[2]) * 1e-3, s_bkwd = (c.phase_ms[1] - p.phase_ms[1]) * 1e-3;
  const double s_rec = (c.phase_ms[3] - p.phase_ms[3] + c.phase_ms[4] - p.phase_ms[4]) * 1e-3;
  const double s_ftle = (c.phase_ms[5] - p.phase_ms[5]) * 1e-3, s_lcs = (c.phase_ms[6] - p.phase_ms[6]) * 1e-3;
  const long long n_fwd = c.integrations_fwd - p.integrations_fwd, n_bkwd = c.integrations_bkwd - p.integrations_bkwd;
  I.total_sim += std::chrono::duration<double>(now - I.t_last).count();
  I.total_lcs += s_lcs;
  I.fwd += s_fwd;
  I.bkwd += s_bkwd;
  I.reconstruct += s_rec;
  I.ftle += s_ftle;
  I.fwd_n += n_fwd;
  I.bkwd_n += n_bkwd;
  I.fwd_s += s_fwd;
  I.bkwd_s += s_bkwd;
  I.t_last = now;
  I.prev = c;
  char a[32], b[32];
  auto es = [](double v, char *out) {
    cfd2lcs::format_es(v, 18, 4, out);
    out[18] = 0;
  };
  auto row = [&](const char *label, double t) {
    es(t, a);
    std::printf("%s%s | %17.4f%% |\n", label, a, I.total_sim > 0 ? t / I.total_sim * 100.0 : 0.0);
  };
  auto rate = [&](const char *label, long long n, double t) {
    es((double)n, a);
    es(t > 0 ? (double)n / t : 0.0, b);
    std::printf("%s%s | %s |\n", label, a, b);
  };
  std::printf("%s\n", lib.sync_timer ? "-----libcfd2lcs CPU overhead (MPI synchronized)-------------------"
                                     : "-----libcfd2lcs CPU overhead (NOT synchronized, rank 0 only)------");
  std::printf("|      TASK             |  WALL CLOCK [SEC] |     %% OF TOTAL     |\n");
  es(I.total_sim, a);
  std::printf("|Application, Total:    |%s |          -         |\n", a);
  row("|cfd2lcs, Total:        |", I.total_lcs);
  row("|cfd2lcs, FWD Advect:   |", I.fwd);
  row("|cfd2lcs, BKWD Advect:  |", I.bkwd);
  row("|cfd2lcs, Reconstruct:  |", I.reconstruct);
  row("|cfd2lcs, LP Re-map:    |", 0.0);
  row("|cfd2lcs, I/O:          |", 0.0);
  row("|cfd2lcs, LCS:          |", I.ftle);
  row("|cfd2lcs, Error Check:  |", 0.0);
  row("|cfd2lcs, Other:        |", I.total_lcs - (I.fwd + I.bkwd + I.reconstruct + I.ftle));
  std::printf("| PARTICLE INTEGRATIONS |  NUMBER [N/STEP]  |     RATE [N/SEC]   |\n");
  rate("|Forward (this step):   |", n_fwd, s_fwd);
  rate("|Backward (this step):  |", n_bkwd, s_bkwd);
  rate("|Forward (cumulative):  |", I.fwd_n, I.fwd_s);
  rate("|Backward (cumulative): |", I.bkwd_n, I.bkwd_s);
  std::printf("------------------------------------------------------------------\n");
  std::fflush(stdout);
}

void do_update(const int *n, const lcsdata_t *u, const lcsdata_t *v, const lcsdata_t *w, lcsdata_t time, bool dev) {
  Library &lib = L();
  if (lib.error) return;
  if (!lib.inited) {
    latch("update: received velocity array of incorrect dimension (cfd2lcs_init was not called)");
    return;
  }
  std::string msg;
  if (!lib.eng->update(n, u, v, w, time, dev, msg)) latch(msg);
  print_info();
}

// cfd2lcs_set_option, src/cfd2lcs.f90:436-622
void do_set_option(const std::string &opt, int val) {
  Library &lib = L();
  if (lib.error) return;
  const bool tf = (val == LCS_TRUE || val == LCS_FALSE);
  bool ok = true;
  if (opt == "SYNCTIMER" || opt == "DEBUG") {
    ok = tf;  // timing / verbosity switches: accepted, no effect on the results
    if (ok && opt == "SYNCTIMER") lib.sync_timer = val == LCS_TRUE;
  } else if (opt == "WRITE_FLOWMAP" || opt == "WRITE_VELOCITY" || opt == "WRITE_BCFLAG") {
    ok = tf;  // variables of the output files (src/cfd2lcs.f90:494-531)
    if (ok) (opt == "WRITE_FLOWMAP" ? lib.opt.write_flowmap : opt == "WRITE_VELOCITY" ? lib.opt.write_velocity : lib.opt.write_bcflag) = val;
  } else if (opt == "WRITE_LCS" || opt == "WRITE_LCS_ASYNC") {  // extensions: output files on / background completion
    ok = tf;
    if (ok) (opt == "WRITE_LCS" ? lib.opt.write_lcs : lib.opt.write_lcs_async) = val;
  } else if (opt == "VELOCITY_INVARIANTS") {
    ok = tf;
    if (ok) lib.opt.velocity_invariants = val;
  } else if (opt == "INCOMPRESSIBLE") {
    ok = tf;
    if (ok) lib.opt.incompressible = val;
  } else if (opt == "AUX_GRID") {
    ok = tf;  // read by cfd2lcs_diagnostic_init (the auxiliary sets are made there) and at each frame
    if (ok) lib.opt.aux_grid = val;
  } else if (opt == "UPDATE_FREQ") {
    ok = true;
  } else if (opt == "INTERPOLATOR") {
    ok = val == NEAREST_NBR || val == LINEAR || val == QUADRATIC || val == CUBIC || val == TSE || val == TSE_LIMIT;
    lib.opt.interpolator = val;  // assigned even for a bad value, as the reference does (:584)
  } else if (opt == "INTEGRATOR") {
    ok = val >= EULER && val <= RK4;
    lib.opt.integrator = val;
  } else if (opt == "MIXED_PRECISION") {  // extension: FP32 velocity data, FP64 positions and flow maps
    ok = tf;
    if (ok && lib.inited) {
      latch("MIXED_PRECISION must be set before cfd2lcs_init");
      return;
    }
    if (ok) lib.opt.mixed_precision = val;
  } else {
    ok = false;
  }
  if (!ok) latch("ERROR, bad libcfd2lcs option/val combination: " + opt + "," + std::to_string(val));
}

// cfd2lcs_set_param, src/cfd2lcs.f90:624-682
void do_set_param(const std::string &p, lcsdata_t val) {
  Library &lib = L();
  if (lib.error) return;
  if (p == "CFL") lib.opt.cfl = (double)val;
  else if (p == "TRACER_INJECT_X") lib.opt.tracer_x = (double)val;
  else if (p == "TRACER_INJECT_Y") lib.opt.tracer_y = (double)val;
  else if (p == "TRACER_INJECT_Z") lib.opt.tracer_z = (double)val;
  else if (p == "TRACER_INJECT_RADIUS") lib.opt.tracer_r = (double)val;
  else latch("ERROR, unknown libcfd2lcs parameter: " + p);
}

}  // namespace

// ----------------------------------------------------------------------- C interface
CFD2LCS_EXPORT void cfd2lcs_init_c(intptr_t usercomm, int n[3], int offset[3], lcsdata_t *x, lcsdata_t *y, lcsdata_t *z, int *flag) {
  (void)usercomm;  // MPI_Comm by value (int or pointer, depending on the MPI); one rank
  do_init(n, offset, x, y, z, flag);
}

CFD2LCS_EXPORT int cfd2lcs_diagnostic_init_c(int lcs_type, int resolution, lcsdata_t t, lcsdata_t h, char label[]) {
  return do_diagnostic_init(lcs_type, resolution, t, h, label);
}

CFD2LCS_EXPORT void cfd2lcs_update_c(int n[3], lcsdata_t *u, lcsdata_t *v, lcsdata_t *w, lcsdata_t time) {
  do_update(n, u, v, w, time, false);
}

CFD2LCS_EXPORT void cfd2lcs_diagnostic_destroy_c(int lcs_handle) {
  (void)lcs_handle;  // a no-op in the reference (src/cfd2lcs.f90:360-386)
}

CFD2LCS_EXPORT void cfd2lcs_set_option_c(char option[], int val) { do_set_option(fstr(option, std::strlen(option)), val); }

CFD2LCS_EXPORT void cfd2lcs_set_param_c(char param[], lcsdata_t val) { do_set_param(fstr(param, std::strlen(param)), val); }

// ----------------------------------------------------------------------- Fortran interface
CFD2LCS_EXPORT void cfd2lcs_init_(int *cfdcomm, int *n, int *offset, lcsdata_t *x, lcsdata_t *y, lcsdata_t *z, int *flag) {
  (void)cfdcomm;
  do_init(n, offset, x, y, z, flag);
}

CFD2LCS_EXPORT void cfd2lcs_diagnostic_init_(int *lcs_handle, int *lcs_type, int *resolution, lcsdata_t *T, lcsdata_t *h, char *label,
                                             size_t label_len) {
  const std::string lab = fstr(label, label_len);
  const int id = do_diagnostic_init(*lcs_type, *resolution, *T, *h, lab.c_str());
  if (lcs_handle) *lcs_handle = id;
}

CFD2LCS_EXPORT void cfd2lcs_update_(int *n, lcsdata_t *ux, lcsdata_t *uy, lcsdata_t *uz, lcsdata_t *time) {
  do_update(n, ux, uy, uz, *time, false);
}

CFD2LCS_EXPORT void cfd2lcs_diagnostic_destroy_(int *lcs_handle) { (void)lcs_handle; }

CFD2LCS_EXPORT void cfd2lcs_set_option_(char *option, int *val, size_t len) { do_set_option(fstr(option, len), *val); }

CFD2LCS_EXPORT void cfd2lcs_set_param_(char *param, lcsdata_t *val, size_t len) { do_set_param(fstr(param, len), *val); }

CFD2LCS_EXPORT void cfd2lcs_finalize_(void) {
  Library &lib = L();
  if (lib.error) return;
  lib.eng.reset();
  lib.inited = false;
}

// ----------------------------------------------------------------------- extensions
CFD2LCS_EXPORT void cfd2lcs_finalize_c(void) { cfd2lcs_finalize_(); }

CFD2LCS_EXPORT int cfd2lcs_get_error_c(char *msg, size_t len) {
  Library &lib = L();
  if (!lib.error && lib.eng) {
    std::string m;
    if (!lib.eng->sync_errors(m)) latch(m);
  }
  if (msg && len > 0) {
    std::strncpy(msg, lib.msg.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  return lib.error;
}

CFD2LCS_EXPORT void cfd2lcs_reset_c(void) {
  Library &lib = L();
  lib.eng.reset();
  lib.inited = false;
  lib.error = 0;
  lib.msg.clear();
  lib.opt = Options();
  lib.sync_timer = false;
  lib.info = InfoState();
}

CFD2LCS_EXPORT int cfd2lcs_get_ftle_c(int lcs_handle, lcsdata_t *ftle) {
  Library &lib = L();
  if (!lib.eng) return 1;
  std::string m;
  return lib.eng->get_ftle(lcs_handle, ftle, m) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_get_flowmap_c(int lcs_handle, lcsdata_t *fm) {
  Library &lib = L();
  if (!lib.eng) return 1;
  std::string m;
  return lib.eng->get_flowmap(lcs_handle, fm, m) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_get_invariants_c(int lcs_handle, lcsdata_t *inv) {
  Library &lib = L();
  if (!lib.eng) return 1;
  std::string m;
  return lib.eng->get_invariants(lcs_handle, inv, m) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_diagnostic_size_c(int lcs_handle, int n[3]) {
  Library &lib = L();
  if (!lib.eng || !n) return 1;
  return lib.eng->diagnostic_size(lcs_handle, n) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_tracer_count_c(int lcs_handle) {
  Library &lib = L();
  return lib.eng ? lib.eng->tracer_count(lcs_handle) : -1;
}

CFD2LCS_EXPORT int cfd2lcs_get_tracers_c(int lcs_handle, lcsdata_t *xyz) {
  Library &lib = L();
  if (!lib.eng || !xyz) return 1;
  std::string m;
  return lib.eng->get_tracers(lcs_handle, xyz, m) ? 0 : 1;
}

CFD2LCS_EXPORT void cfd2lcs_update_device_c(int n[3], const lcsdata_t *d_u, const lcsdata_t *d_v, const lcsdata_t *d_w, lcsdata_t time) {
  do_update(n, d_u, d_v, d_w, time, true);
}

CFD2LCS_EXPORT const lcsdata_t *cfd2lcs_ftle_device_ptr_c(int lcs_handle) {
  Library &lib = L();
  return lib.eng ? lib.eng->ftle_device_ptr(lcs_handle) : nullptr;
}

CFD2LCS_EXPORT void cfd2lcs_get_counters_c(long long c[8]) {
  Library &lib = L();
  const Counters &k = lib.eng ? lib.eng->counters() : lib.zero;
  c[0] = k.integrations_fwd;
  c[1] = k.integrations_bkwd;
  c[2] = k.nsub_fwd;
  c[3] = k.nsub_bkwd;
  c[4] = k.ftle_frames;
  c[5] = k.updates;
  c[6] = k.kernel_launches;
  c[7] = k.slots_composed;
}

CFD2LCS_EXPORT void cfd2lcs_get_phase_times_c(double t[7]) {
  Library &lib = L();
  const Counters &k = lib.eng ? lib.eng->counters() : lib.zero;
  for (int q = 0; q < 7; q++) t[q] = k.phase_ms[q];
}

// Event-timed hot kernels: t[0] backward SL subcycle kernels (ms, cumulative),
// t[1] forward particle kernels; n[0], n[1] their launch counts.
CFD2LCS_EXPORT void cfd2lcs_get_kernel_times_c(double t[2], long long n[2]) {
  Library &lib = L();
  const Counters &k = lib.eng ? lib.eng->counters() : lib.zero;
  t[0] = k.sl_kernel_ms;
  t[1] = k.fwd_kernel_ms;
  n[0] = k.sl_kernel_launches;
  n[1] = k.fwd_kernel_launches;
}

// Launches of the kernels that stage their spline taps in shared memory: n[0] backward
// semi-Lagrangian subcycles, n[1] forward particle subcycles (cumulative).
CFD2LCS_EXPORT void cfd2lcs_get_staged_launches_c(long long n[2]) {
  Library &lib = L();
  const Counters &k = lib.eng ? lib.eng->counters() : lib.zero;
  n[0] = k.sl_staged_launches;
  n[1] = k.fwd_staged_launches;
}

// Of the staged backward launches, those of the LINEAR kernel that marches planes along z
// (cumulative).
CFD2LCS_EXPORT void cfd2lcs_get_march_launches_c(long long *n) {
  Library &lib = L();
  const Counters &k = lib.eng ? lib.eng->counters() : lib.zero;
  *n = k.sl_march_launches;
}

// The engine's choice between staged and gathering subcycle kernels: choice[f] for the backward
// (f = 0) and forward (f = 1) kernel, -1 while sampling or where staging does not apply, 0
// gathering, 1 staged; ms[2f], ms[2f+1] the mean launch times measured for the two.
CFD2LCS_EXPORT void cfd2lcs_get_tuning_c(int choice[2], double ms[4]) {
  Library &lib = L();
  for (int f = 0; f < 2; f++) choice[f] = -1;
  for (int q = 0; q < 4; q++) ms[q] = 0.0;
  if (lib.eng) lib.eng->tuning(choice, ms);
}

// Host-only formatting hook (no device work): the Fortran ESw.d editing the output files use,
// for checking the writer on machines without a GPU.  out receives w characters and a NUL.
CFD2LCS_EXPORT void cfd2lcs_b200_format_es(double v, int w, int d, char *out) {
  if (!out || w <= 0 || w > 60) return;
  cfd2lcs::format_es(v, w, d, out);
  out[w] = 0;
}

// Host-only grid set-up (no device work): the padded coordinates, flags, boundary normals
// and inverse half spans the library derives at init.  Used to check the host logic on
// machines without a GPU.  Returns 0 on success.
CFD2LCS_EXPORT int cfd2lcs_b200_grid_tables(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                                            lcsdata_t *xyz_pad, int *flag_pad, lcsdata_t *nrm_pad, lcsdata_t *inv_delta, int *per,
                                            char *msg, size_t len) {
  Options o;
  std::unique_ptr<EngineBase> e = cfd2lcs::make_engine(&o);
  std::string m;
  const bool ok = e->host_grid_tables(n, x, y, z, flag, xyz_pad, flag_pad, nrm_pad, inv_delta, per, m);
  if (msg && len > 0) {
    std::strncpy(msg, m.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  return ok ? 0 : 1;
}

// Host-only: the least-squares gradient weights the library derives for a non-rectilinear
// grid (compute_lsgw with the six face neighbours, src/gradient_m.f90:114-217), 18 padded
// arrays [neighbour 0..5][derivative 0..2] of (n+2) points each, zero on a rectilinear grid.
// *curv is set to 1 for a non-rectilinear grid.  Returns 0 on success.
CFD2LCS_EXPORT int cfd2lcs_b200_grid_lsq_weights(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z,
                                                 const int *flag, lcsdata_t *w, int *curv, char *msg, size_t len) {
  HostGrid<lcsdata_t> g;
  const bool ok = g.build(n, x, y, z, flag);
  if (msg && len > 0) {
    std::strncpy(msg, ok ? "" : g.error.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  if (!ok) return 1;
  const size_t nt = (size_t)g.ntot();
  if (curv) *curv = g.P.curv;
  for (size_t q = 0; q < 18 * nt; q++) w[q] = g.lsw.empty() ? lcsdata_t(0) : g.lsw[q];
  return 0;
}

// Allocation-free recomputation of a diagnostic's latest FTLE frame into caller-owned device
// buffers (see include/cfd2lcs_b200.h).  Returns 0 on success; on failure the error is
// latched like any other library error and 1 is returned.
CFD2LCS_EXPORT int cfd2lcs_reconstruct_noalloc_c(int lcs_handle, lcsdata_t *d_ftle, lcsdata_t *d_fm) {
  Library &lib = L();
  if (lib.error) return 1;
  if (!lib.eng) {
    latch("reconstruct_noalloc: cfd2lcs_init was not called");
    return 1;
  }
  std::string msg;
  if (!lib.eng->reconstruct_noalloc(lcs_handle, d_ftle, d_fm, msg)) {
    latch(msg);
    return 1;
  }
  return 0;
}

// ----------------------------------------------------------------------- batched form
// Many independent instances -- each with its own grid, options and diagnostics -- advanced
// together.  An update of the batch runs update_begin for every listed instance (ingest + CFL
// read-back, each instance on its own stream), then update_enqueue for every instance, then
// update_collect: one host wait per instance for its CFL number, and the instances' kernels
// overlap on the device.  The batch has its own error state (cfd2lcs_batch_error_c) and does
// not touch the single instance of the reference API.
namespace {

struct BatchInstance {
  Options opt;  // the engine keeps a pointer to it
  std::unique_ptr<EngineBase> eng;
  int n[3];
};

struct Batch {
  std::vector<std::unique_ptr<BatchInstance>> inst;
  int error = 0;
  std::string msg;
};

Batch &BT() {
  static Batch b;
  return b;
}

int batch_fail(const std::string &m) {
  Batch &b = BT();
  if (!b.error) b.msg = m;
  b.error = 1;
  return -1;
}

int batch_fail_rc(const std::string &m) {
  batch_fail(m);
  return 1;
}

BatchInstance *batch_get(int id) {
  Batch &b = BT();
  if (id < 0 || id >= (int)b.inst.size()) return nullptr;
  return b.inst[id].get();
}

}  // namespace

CFD2LCS_EXPORT int cfd2lcs_batch_add_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                                       int integrator, int interpolator, lcsdata_t cfl, int mixed_precision) {
  Batch &b = BT();
  if (b.error) return -1;
  if (integrator < EULER || integrator > RK4) return batch_fail("batch_add: bad integrator");
  if (interpolator != NEAREST_NBR && interpolator != LINEAR && interpolator != QUADRATIC && interpolator != CUBIC && interpolator != TSE &&
      interpolator != TSE_LIMIT)
    return batch_fail("batch_add: bad interpolator");
  if (!(cfl > lcsdata_t(0))) return batch_fail("batch_add: CFL must be positive");
  std::unique_ptr<BatchInstance> bi(new BatchInstance());
  bi->opt.integrator = integrator;
  bi->opt.interpolator = interpolator;
  bi->opt.cfl = (double)cfl;
  bi->opt.mixed_precision = mixed_precision ? 1 : 0;
  bi->opt.shared_device = 1;
  for (int a = 0; a < 3; a++) bi->n[a] = n[a];
  bi->eng = cfd2lcs::make_engine(&bi->opt);
  std::string msg;
  if (!bi->eng->init(n, x, y, z, flag, msg)) return batch_fail("batch_add: " + msg);
  b.inst.push_back(std::move(bi));
  return (int)b.inst.size() - 1;
}

CFD2LCS_EXPORT int cfd2lcs_batch_diagnostic_init_c(int id, int lcs_type, lcsdata_t T, lcsdata_t h) {
  Batch &b = BT();
  if (b.error) return -1;
  BatchInstance *bi = batch_get(id);
  if (!bi) return batch_fail("batch_diagnostic_init: unknown instance");
  std::string msg;
  const int hd = bi->eng->diagnostic_init(lcs_type, 0, T, h, "batch", msg);
  if (hd < 0) return batch_fail("batch_diagnostic_init: " + msg);
  return hd;
}

CFD2LCS_EXPORT int cfd2lcs_batch_update_device_c(int count, const int *ids, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                                                 const lcsdata_t *const *d_w, const lcsdata_t *time) {
  Batch &b = BT();
  if (b.error) return 1;
  std::vector<BatchInstance *> run;
  for (int q = 0; q < count; q++) {
    BatchInstance *bi = batch_get(ids[q]);
    if (!bi) return batch_fail_rc("batch_update: unknown instance");
    run.push_back(bi);
  }
  std::string msg;
  for (int q = 0; q < count; q++)
    if (!run[q]->eng->update_begin(run[q]->n, d_u[q], d_v[q], d_w[q], time[q], true, msg)) return batch_fail_rc(msg);
  for (int q = 0; q < count; q++)
    if (!run[q]->eng->update_enqueue(msg)) return batch_fail_rc(msg);
  for (int q = 0; q < count; q++)
    if (!run[q]->eng->update_collect(msg)) return batch_fail_rc(msg);
  return 0;
}

CFD2LCS_EXPORT int cfd2lcs_batch_get_ftle_c(int id, int lcs_handle, lcsdata_t *ftle) {
  BatchInstance *bi = batch_get(id);
  if (!bi) return 1;
  std::string m;
  return bi->eng->get_ftle(lcs_handle, ftle, m) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_batch_get_flowmap_c(int id, int lcs_handle, lcsdata_t *fm) {
  BatchInstance *bi = batch_get(id);
  if (!bi) return 1;
  std::string m;
  return bi->eng->get_flowmap(lcs_handle, fm, m) ? 0 : 1;
}

CFD2LCS_EXPORT int cfd2lcs_batch_get_counters_c(int id, long long c[8]) {
  BatchInstance *bi = batch_get(id);
  if (!bi) return 1;
  const Counters &k = bi->eng->counters();
  c[0] = k.integrations_fwd;
  c[1] = k.integrations_bkwd;
  c[2] = k.nsub_fwd;
  c[3] = k.nsub_bkwd;
  c[4] = k.ftle_frames;
  c[5] = k.updates;
  c[6] = k.kernel_launches;
  c[7] = k.slots_composed;
  return 0;
}

CFD2LCS_EXPORT int cfd2lcs_batch_size_c(void) { return (int)BT().inst.size(); }

CFD2LCS_EXPORT int cfd2lcs_batch_error_c(char *msg, size_t len) {
  Batch &b = BT();
  if (msg && len > 0) {
    std::strncpy(msg, b.msg.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  return b.error;
}

CFD2LCS_EXPORT void cfd2lcs_batch_reset_c(void) {
  Batch &b = BT();
  b.inst.clear();
  b.error = 0;
  b.msg.clear();
}

// ----------------------------------------------------------------------- adjoint
// Gradient of J = sum weight * FTLE (backward FTLE of the whole horizon) with respect to the
// velocity at every level; see include/cfd2lcs_b200.h.  Returns 0, or 1 with msg.
CFD2LCS_EXPORT int cfd2lcs_adjoint_ftle_interp_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                                                 int integrator,
                                                 int interpolator, lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u,
                                                 const lcsdata_t *const *d_v, const lcsdata_t *const *d_w, const lcsdata_t *times,
                                                 const lcsdata_t *d_weight, int checkpoint_every, double *J, lcsdata_t *const *d_gu,
                                                 lcsdata_t *const *d_gv, lcsdata_t *const *d_gw, char *msg, size_t len) {
  cfd2lcs::AdjointProblem p{n, x, y, z, integrator, (double)cfl, nlevels, d_u, d_v, d_w, times, d_weight, checkpoint_every,
                            d_gu, d_gv, d_gw};
  p.interpolator = interpolator;
  p.flag = flag;
  std::string m;
  const bool ok = cfd2lcs::adjoint_ftle(p, J, m);
  if (msg && len > 0) {
    std::strncpy(msg, m.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  return ok ? 0 : 1;
}

// The same with LINEAR interpolation.
CFD2LCS_EXPORT int cfd2lcs_adjoint_ftle_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, int integrator,
                                          lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                                          const lcsdata_t *const *d_w, const lcsdata_t *times, const lcsdata_t *d_weight,
                                          int checkpoint_every, double *J, lcsdata_t *const *d_gu, lcsdata_t *const *d_gv,
                                          lcsdata_t *const *d_gw, char *msg, size_t len) {
  return cfd2lcs_adjoint_ftle_interp_c(n, x, y, z, nullptr, integrator, LINEAR, cfl, nlevels, d_u, d_v, d_w, times, d_weight, checkpoint_every, J,
                                       d_gu, d_gv, d_gw, msg, len);
}

// Tangent-linear check of the adjoint: J and dJ = <dJ/du, d> for one direction d, by a forward-
// mode sweep alongside the flow map; see include/cfd2lcs_b200.h.  Returns 0, or 1 with msg.
CFD2LCS_EXPORT int cfd2lcs_tangent_ftle_interp_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag,
                                                 int integrator,
                                                 int interpolator, lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u,
                                                 const lcsdata_t *const *d_v, const lcsdata_t *const *d_w, const lcsdata_t *times,
                                                 const lcsdata_t *d_weight, const lcsdata_t *const *d_du, const lcsdata_t *const *d_dv,
                                                 const lcsdata_t *const *d_dw, double *J, double *dJ, char *msg, size_t len) {
  std::string m;
  bool ok = d_du && d_dv && d_dw && dJ;
  if (!ok) m = "tangent: a direction (d_du, d_dv, d_dw) and dJ are required";
  if (ok) {
    cfd2lcs::AdjointProblem p{n, x, y, z, integrator, (double)cfl, nlevels, d_u, d_v, d_w, times, d_weight, 1, nullptr, nullptr, nullptr};
    p.du = d_du;
    p.dv = d_dv;
    p.dw = d_dw;
    p.dJ = dJ;
    p.interpolator = interpolator;
    p.flag = flag;
    ok = cfd2lcs::adjoint_ftle(p, J, m);
  }
  if (msg && len > 0) {
    std::strncpy(msg, m.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  return ok ? 0 : 1;
}

// The same with LINEAR interpolation.
CFD2LCS_EXPORT int cfd2lcs_tangent_ftle_c(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, int integrator,
                                          lcsdata_t cfl, int nlevels, const lcsdata_t *const *d_u, const lcsdata_t *const *d_v,
                                          const lcsdata_t *const *d_w, const lcsdata_t *times, const lcsdata_t *d_weight,
                                          const lcsdata_t *const *d_du, const lcsdata_t *const *d_dv, const lcsdata_t *const *d_dw,
                                          double *J, double *dJ, char *msg, size_t len) {
  return cfd2lcs_tangent_ftle_interp_c(n, x, y, z, nullptr, integrator, LINEAR, cfl, nlevels, d_u, d_v, d_w, times, d_weight, d_du, d_dv, d_dw, J,
                                       dJ, msg, len);
}
