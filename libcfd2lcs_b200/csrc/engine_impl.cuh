// Host orchestration of the device path: init (grid tables to HBM), diagnostic init,
// and the per-update sequence of cfd2lcs_update (src/cfd2lcs.f90:55-250).
#pragma once

#include "engine.h"

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <map>
#include <mutex>
#include <array>

#include <cuda.h>

#include "grid.h"
#include "kernels.cuh"
#include "tile.cuh"
#include "spline_host.h"
#include "writer.h"

namespace cfd2lcs {

namespace {

enum { FTLE_FWD = 0, FTLE_BKWD = 1, LP_TRACER = 2 };
enum { NEAREST_NBR = 0, LINEAR = 1, QUADRATIC = 2, CUBIC = 3, TSE = 5, TSE_LIMIT = 6 };

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      msg = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " + #call;               \
      return false;                                                                              \
    }                                                                                            \
  } while (0)

// Fortran NINT
inline long fnint(double v) { return v >= 0 ? (long)std::floor(v + 0.5) : -(long)std::floor(-v + 0.5); }

// Device allocations released together with the engine.
class DevArena {
 public:
  ~DevArena() { release(); }
  void release() {
    for (void *p : ptrs_) cudaFree(p);
    ptrs_.clear();
  }
  // Every buffer gets 256 bytes of slack past its end: the staged-tile kernels copy rows in
  // whole 16-byte units, so the copy of an array's last row may read up to 15 bytes past it.
  template <typename X>
  X *alloc(size_t n, std::string &msg) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(X) + 256);
    if (e != cudaSuccess) {
      msg = std::string("device allocation failed: ") + cudaGetErrorString(e);
      return nullptr;
    }
    ptrs_.push_back(p);
    return static_cast<X *>(p);
  }

 private:
  std::vector<void *> ptrs_;
};

template <typename T>
struct SplineSet {
  int deg = 0;
  SplineAxes<T> axes{};
};

// The lcs grid of a diagnostic with resolution /= 0 (new_sgrid_from_sgrid, src/sgrid_m.f90:
// 446-761): its host set-up and device tables, each lcs node's position and solver-grid node
// after tracking to the solver grid (init_lp + track_lp2node), and, for backward sets, the
// working copy of those nodes (set_lp_bc clamps them in place during the updates).
template <typename T>
struct LcsGrid {
  HostGrid<lcsdata_t> hg;
  DevGrid<T> dg{};
  long N = 0, ntot = 0;
  T *pos[3] = {nullptr, nullptr, nullptr};
  int *nos_reset[3] = {nullptr, nullptr, nullptr};
  int *nos[3] = {nullptr, nullptr, nullptr};
  SplineSet<T> sp[4];  // B-spline axes of the lcs grid by degree (flow-map fits and samples)
  // output files: coordinate lines and interior flags; lp%ugrid (the frame's velocity at the
  // nodes, T) and the padded snapshot / its coefficients it is sampled from (solver grid, TV)
  std::shared_ptr<const std::vector<double>> out_lines[3];
  std::shared_ptr<const std::vector<int8_t>> out_flags;
  T *ugrid[3] = {nullptr, nullptr, nullptr};
};

template <typename T, typename TV>
struct Diag {
  int handle = 0, type = 0;
  std::string label;  // lcs%label: names the output files
  lcsdata_t T_ = 0, h = 0, dt_factor = 1;
  int nslot = 0;
  // backward: working flow map (double buffered, padded)
  T *fm[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int cur = 0;
  T *fmcoef[3] = {nullptr, nullptr, nullptr};
  // forward: particles (P current, P2 the target of the re-sort by grid cell) and the
  // counting sort's keys, cell counts, offsets and chunk sums
  Particles<T> P{}, P2{};
  unsigned *pkey = nullptr;
  int *pcnt = nullptr, *poffs = nullptr, *ptsum = nullptr;
  SortTiles sort_geom{};  // cell tiles of the last sort (the staged forward kernel reads one tile per block)
  int fwd_variant = 0;    // forward kernel until the next sort: 0 gathering, 1 staged
  long since_sort = 1L << 40;  // forward subcycles since the particles were last sorted (or reset)
  // event-timed cost of the last sort, launch time right after it, and the launch time lost
  // since then (gathering forward kernels: the re-sort schedule of sort_due)
  double sort_ms = 0, base_ms = -1, excess_ms = 0;
  // ring of sub-flow maps (padded) and their spline coefficients
  std::vector<T *> slot;      // 3 per slot
  std::vector<T *> slotcoef;  // 3 per slot (allocated on first spline use)
  std::vector<int> written, coef_deg;
  T **slot_list_dev = nullptr;  // pointers of the slots used by one composition
  std::vector<T *> slot_list_host;
  std::vector<int> last_order;  // slots composed by the latest frame, in order
  // time-blended spline coefficients of the stage velocities (B-spline interpolators)
  TV *blend[3][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  double blend_ct[3] = {-1, -1, -1};
  long long blend_update[3] = {-1, -1, -1};
  T *composed[3] = {nullptr, nullptr, nullptr};  // interior, last FTLE frame
  lcsdata_t *ftle = nullptr;                      // interior
  lcsdata_t *inv[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // velocity invariants (interior)
  bool have_frame = false;
  // LP_TRACER: particles in P (np of them), time advected, and whether they still move
  // (destroy_lp once the lifetime exceeds T, src/cfd2lcs.f90:225-231)
  int np = 0;
  lcsdata_t lifetime = 0;
  bool active = true;
  std::shared_ptr<LcsGrid<T>> lg;  // refined / coarsened lcs grid (null: the solver grid)
  // AUX_GRID: an auxiliary set (aux_parent = index + 1 of its diagnostic in the engine's list,
  // handle 0), or a diagnostic's six sets X0, Y0, Z0, X1, Y1, Z1 (indices) and the per-node
  // separations of each pair
  int aux_parent = 0;
  std::vector<int> aux;
  T *auxden[3] = {nullptr, nullptr, nullptr};
};

}  // namespace

// cuTensorMapEncodeTiled of the driver, looked up once through the runtime's entry-point query
// (the library links the runtime statically and no driver library); null where unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                   const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled_fn() {
  static const EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// The allocation-free entry point's table of sub-flow-map pointers (engine.cu): its size (in
// sub-flow maps) and its device address on device dev.
#define NOALLOC_MAX_SUBMAPS 256
bool noalloc_table_address(int dev, void **out, std::string &msg);

// TV: storage type of the velocity levels, their spline coefficients and the blended stage
// coefficients (FP32 in the mixed-precision form).  Positions, flow maps, sub-flow maps,
// composition and FTLE stay in the interface type T = lcsdata_t.
template <typename TV>
class Engine : public EngineBase {
  using T = lcsdata_t;
  using DiagT = Diag<T, TV>;

 public:
  explicit Engine(const Options *opt) : opt_(opt) {}
  ~Engine() override {
    writer_.reset();  // finishes the queued files while their staged copies' stream still exists
    if (stream_) cudaStreamSynchronize(stream_);
    arena_.release();
    for (auto &e : ev_) cudaEventDestroy(e);
    for (auto &e : evpool_) cudaEventDestroy(e);
    if (red_host_) cudaFreeHost(red_host_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  bool host_grid_tables(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag, lcsdata_t *xyz,
                        int *flag_pad, lcsdata_t *nrm, lcsdata_t *invd, int *per, std::string &msg) override {
    HostGrid<lcsdata_t> g;
    if (!g.build(n, x, y, z, flag)) {
      msg = g.error;
      return false;
    }
    const long nt = g.ntot();
    for (int k = 0; k <= n[2] + 1; k++)
      for (int j = 0; j <= n[1] + 1; j++)
        for (int i = 0; i <= n[0] + 1; i++) {
          const long p = g.pidx(i, j, k);
          for (int c = 0; c < 3; c++) {
            if (xyz) xyz[c * nt + p] = g.coord(c, i, j, k);
            if (nrm) nrm[c * nt + p] = g.bcnorm.empty() ? lcsdata_t(0) : g.bcnorm[(size_t)c * nt + p];
          }
          if (flag_pad) flag_pad[p] = g.flag.empty() ? 0 : g.flag[p];
          if (invd) {
            const bool inside = i >= 1 && j >= 1 && k >= 1 && i <= n[0] && j <= n[1] && k <= n[2];
            const int idx[3] = {i, j, k};
            for (int a = 0; a < 3; a++) {
              lcsdata_t v = 0;
              if (inside && g.P.curv) {
                v = g.invdp[a][p];
              } else if (inside) {
                const int b = (a + 1) % 3, c = (a + 2) % 3;
                const int cb = (idx[b] - 1 == 0 ? 1 : 0) | (idx[b] + 1 == n[b] + 1 ? 2 : 0);
                const int cc = (idx[c] - 1 == 0 ? 1 : 0) | (idx[c] + 1 == n[c] + 1 ? 2 : 0);
                v = g.invd[a][((size_t)idx[a] * 4 + cb) * 4 + cc];
              }
              invd[a * nt + p] = v;
            }
          }
        }
    if (per)
      for (int a = 0; a < 3; a++) per[a] = g.P.per[a];
    return true;
  }

  bool init(const int n[3], const lcsdata_t *x, const lcsdata_t *y, const lcsdata_t *z, const int *flag, std::string &msg) override {
    if (!hg_.build(n, x, y, z, flag)) {
      msg = hg_.error;
      return false;
    }
    CK(cudaGetDevice(&dev_));  // the device this engine's stream and buffers live on
    CK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev_));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (int e = 0; e < 10; e++) {
      cudaEvent_t ev;
      CK(cudaEventCreate(&ev));
      ev_.push_back(ev);
    }
    CK(cudaMallocHost(&red_host_, sizeof(DevReduce)));
    if (const char *e = std::getenv("CFD2LCS_B200_LINEAR_BLEND_MIN")) lin_blend_min_ = std::atol(e);
    if (const char *e = std::getenv("CFD2LCS_B200_TMA_TENSOR")) tma_tensor_ = std::atoi(e) != 0;
    if (const char *e = std::getenv("CFD2LCS_B200_COMPOSE_SORT_MIN")) compose_sort_min_ = std::atol(e);
    if (const char *e = std::getenv("CFD2LCS_B200_COMPOSE_SORT_EVERY")) compose_sort_every_ = std::max(1, std::atoi(e));
    if (const char *e = std::getenv("CFD2LCS_B200_COMPOSE_MINB")) compose_minb_ = std::atoi(e) >= 4 ? 4 : 2;
    if (const char *e = std::getenv("CFD2LCS_B200_SL_TILE")) tile_mode_ = std::max(0, std::min(2, std::atoi(e)));
    if (const char *e = std::getenv("CFD2LCS_B200_SL_MARCH")) sl_march_ = std::atoi(e) != 0;
    if (const char *e = std::getenv("CFD2LCS_B200_SORT_EVERY")) sort_every_ = std::max(0, std::atoi(e));
    if (const char *e = std::getenv("CFD2LCS_B200_SL_MARCH_KC")) sl_march_kc_ = std::max(0, std::atoi(e));
    for (int a = 0; a < 3; a++) n_[a] = n[a];
    // coordinate lines (and, on a non-rectilinear grid, the node coordinates) and interior flags
    // for the output files
    for (int a = 0; a < 3; a++) {
      out_lines_[a] = std::make_shared<std::vector<double>>(hg_.lt[a].begin() + 1, hg_.lt[a].begin() + 1 + n[a]);
      if (hg_.P.curv) {
        auto c = std::make_shared<std::vector<double>>();
        c->reserve((size_t)n[0] * n[1] * n[2]);
        for (int k = 1; k <= n[2]; k++)
          for (int j = 1; j <= n[1]; j++)
            for (int i = 1; i <= n[0]; i++) c->push_back((double)hg_.coord(a, i, j, k));
        out_coords_[a] = c;
      }
    }
    {
      auto fl = std::make_shared<std::vector<int8_t>>((size_t)n[0] * n[1] * n[2]);
      for (size_t q = 0; q < fl->size(); q++) (*fl)[q] = (int8_t)flag[q];
      out_flags_ = fl;
    }
    N_ = (long)n[0] * n[1] * n[2];
    ntot_ = hg_.ntot();
    // grid tables
    if (!make_dev_grid(hg_, dg_, msg)) return false;
    // velocity levels (zero-initialised, as init_sr1 does, src/structured_m.f90:73-96)
    for (int l = 0; l < 2; l++)
      for (int c = 0; c < 3; c++) {
        if (!(u_[l][c] = arena_.alloc<TV>(ntot_, msg))) return false;
        CK(cudaMemsetAsync(u_[l][c], 0, ntot_ * sizeof(TV), stream_));
      }
    if (!(stage_ = arena_.alloc<lcsdata_t>((size_t)3 * N_, msg))) return false;
    if (!(red_ = arena_.alloc<DevReduce>(1, msg))) return false;
    CK(cudaMemsetAsync(red_, 0, sizeof(DevReduce), stream_));
    CK(cudaStreamSynchronize(stream_));
    first_call_ = true;
    return true;
  }

  int diagnostic_init(int type, int resolution, lcsdata_t Tint, lcsdata_t h, const char *label, std::string &msg) override {
    if (type == LP_TRACER) return tracer_init(Tint, h, label, resolution, msg);
    if (type != FTLE_FWD && type != FTLE_BKWD) {
      msg = "ERROR, bad specification for lcs_type. Options are: FTLE_FWD, FTLE_BKWD, LP_TRACER";
      return -1;
    }
    if (!(h > lcsdata_t(0)) || !(Tint > lcsdata_t(0))) {
      msg = "diagnostic_init: T and h must be positive";
      return -1;
    }
    DiagT d;
    // lcs%sgrid (src/cfd2lcs.f90:302-310); new_sgrid_from_sgrid may reset the resolution to 0
    if (resolution != 0 && !make_lcs_grid(d, type, resolution, msg)) return -1;
    d.handle = ++handle_count_;
    d.type = type;
    d.label = label ? label : "";
    while (!d.label.empty() && d.label.back() == ' ') d.label.pop_back();  // trim(label)
    d.T_ = Tint;
    d.h = h;
    d.dt_factor = type == FTLE_BKWD ? lcsdata_t(1) / lcsdata_t(std::max(1 + resolution, 1)) : lcsdata_t(1);
    d.nslot = (int)std::max(1L, fnint((double)(Tint / h)));
    if (!alloc_diag(d, msg)) return -1;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return fail(msg, "sync");
    const int handle = d.handle;
    diags_.push_back(d);
    // AUX_GRID (init_ftle, src/lcs_m.f90:50-53): six auxiliary particle sets around the nodes
    if (opt_->aux_grid && !create_aux((int)diags_.size() - 1, msg)) return -1;
    return handle;
  }

  // Device buffers of a diagnostic (or auxiliary set) on its grid: working flow maps or
  // particles and their sort tables, the ring of sub-flow maps, the composed map and the FTLE.
  bool alloc_diag(DiagT &d, std::string &msg) {
    const long dn = dN(d), dt = dT(d);
    if (d.type == FTLE_BKWD) {
      for (int b = 0; b < 2; b++)
        for (int c = 0; c < 3; c++) {
          if (!(d.fm[b][c] = arena_.alloc<T>(dt, msg))) return false;
          if (cudaMemsetAsync(d.fm[b][c], 0, dt * sizeof(T), stream_) != cudaSuccess) { msg = "CUDA error in memset"; return false; }
        }
      if (d.lg && !reset_refined_nodes(d, msg)) return false;
    } else {
      for (Particles<T> *Q : {&d.P, &d.P2}) {
        for (int c = 0; c < 3; c++) {
          if (!(Q->x[c] = arena_.alloc<T>(dn, msg))) return false;
          if (!(Q->dx[c] = arena_.alloc<T>(dn, msg))) return false;
          if (!(Q->no[c] = arena_.alloc<int>(dn, msg))) return false;
        }
        if (!(Q->id = arena_.alloc<int>(dn, msg))) return false;
      }
      if (!(d.P.slot = arena_.alloc<int>(dn, msg))) return false;
      d.P2.slot = d.P.slot;  // the inverse map is rewritten whole by every permutation
      // key space for either tile shape of the sort (gathering or staged forward kernel)
      const long ncell = std::max(sort_key_space(sort_tiles(n_, 32, SORT_TY, SORT_TZ)), sort_key_space(sort_tiles(n_, FWT_TX, FWT_TY, FWT_TZ)));
      if (ncell > (long)std::numeric_limits<int>::max()) {
        msg = "diagnostic_init: grid too large for the forward particle sort";
        return false;
      }
      if (!(d.pkey = arena_.alloc<unsigned>(dn, msg))) return false;
      if (!(d.pcnt = arena_.alloc<int>(ncell, msg))) return false;
      if (!(d.poffs = arena_.alloc<int>(ncell, msg))) return false;
      if (!(d.ptsum = arena_.alloc<int>((ncell + SORT_TILE - 1) / SORT_TILE, msg))) return false;
      if (cudaMemsetAsync(d.pcnt, 0, ncell * sizeof(int), stream_) != cudaSuccess) { msg = "CUDA error in memset"; return false; }
      launch_reset(d);
    }
    d.slot.assign((size_t)3 * d.nslot, nullptr);
    d.slotcoef.assign((size_t)3 * d.nslot, nullptr);
    d.written.assign(d.nslot, 0);
    d.coef_deg.assign(d.nslot, 0);
    for (int s = 0; s < 3 * d.nslot; s++)
      if (!(d.slot[s] = arena_.alloc<T>(dt, msg))) return false;
    if (!(d.slot_list_dev = arena_.alloc<T *>((size_t)3 * d.nslot, msg))) return false;
    d.slot_list_host.assign((size_t)3 * d.nslot, nullptr);
    for (int c = 0; c < 3; c++)
      if (!(d.composed[c] = arena_.alloc<T>(dn, msg))) return false;
    if (!(d.ftle = arena_.alloc<lcsdata_t>(dn, msg))) return false;
    if (!d.lg && (d.type == FTLE_FWD || d.type == FTLE_BKWD) && !ensure_compose_scratch(msg)) return false;
    return true;
  }

  // Composition one sub-map at a time with the particles re-sorted between sub-maps (k_compose_step)
  // on grids of at least this many points (the sort costs more than it saves on small grids);
  // CFD2LCS_B200_COMPOSE_SORT_MIN at cfd2lcs_init overrides it (the tests take both paths on
  // small grids).
#ifndef CFD2LCS_COMPOSE_SORT_MIN
#define CFD2LCS_COMPOSE_SORT_MIN (1L << 20)
#endif
  long compose_sort_min_ = CFD2LCS_COMPOSE_SORT_MIN;
  // Re-sort every this many sub-maps, and resident blocks per SM of k_compose_step (2 or 4;
  // CFD2LCS_B200_COMPOSE_SORT_EVERY / _MINB override them).  Measured on B200, ABC 256^3 RK3
  // CUBIC, frames of 10 sub-maps with h = 0.1 (ms per frame): node-ordered k_compose 34.8; steps
  // with 2 blocks, sorted every sub-map 39.5; 4 blocks: every sub-map 35.2, every 2nd 34.2, every
  // 3rd 33.6.  With h = 1 (sub-maps that move points ~120 cells, the ABC 256^3 T = 10 workload)
  // the node-ordered kernel took 72.6 and the steps sorted every sub-map (2 blocks) 69.0.
  int compose_sort_every_ = 2, compose_minb_ = 4;
  // the composition particles of every solver-grid frame (one frame at a time uses them)
  Particles<T> cp_[2]{};
  unsigned *cp_key_ = nullptr;
  int *cp_cnt_ = nullptr, *cp_offs_ = nullptr, *cp_tsum_ = nullptr;

  bool ensure_compose_scratch(std::string &msg) {
    if (N_ < compose_sort_min_ || cp_[0].x[0]) return true;
    for (Particles<T> *Q : {&cp_[0], &cp_[1]}) {
      for (int c = 0; c < 3; c++) {
        if (!(Q->x[c] = arena_.alloc<T>(N_, msg))) return false;
        if (!(Q->dx[c] = arena_.alloc<T>(N_, msg))) return false;
        if (!(Q->no[c] = arena_.alloc<int>(N_, msg))) return false;
      }
      if (!(Q->id = arena_.alloc<int>(N_, msg))) return false;
    }
    if (!(cp_[0].slot = arena_.alloc<int>(N_, msg))) return false;
    cp_[1].slot = cp_[0].slot;
    const long ncell = sort_key_space(sort_tiles(n_, 32, SORT_TY, SORT_TZ));
    if (ncell > (long)std::numeric_limits<int>::max()) {
      msg = "diagnostic_init: grid too large for the composition sort";
      return false;
    }
    if (!(cp_key_ = arena_.alloc<unsigned>(N_, msg))) return false;
    if (!(cp_cnt_ = arena_.alloc<int>(ncell, msg))) return false;
    if (!(cp_offs_ = arena_.alloc<int>(ncell, msg))) return false;
    if (!(cp_tsum_ = arena_.alloc<int>((ncell + SORT_TILE - 1) / SORT_TILE, msg))) return false;
    if (cudaMemsetAsync(cp_cnt_, 0, ncell * sizeof(int), stream_) != cudaSuccess) {
      msg = "CUDA error in memset";
      return false;
    }
    return true;
  }

  bool update(const int n[3], const lcsdata_t *u, const lcsdata_t *v, const lcsdata_t *w, lcsdata_t time, bool device_ptrs,
              std::string &msg) override {
    return update_begin(n, u, v, w, time, device_ptrs, msg) && update_enqueue(msg) && update_collect(msg);
  }

  // First half of an update: time levels, velocity ingest (+ spline fits of the new level)
  // and the asynchronous read-back of the CFL maximum.  Returns without waiting.
  bool update_begin(const int n[3], const lcsdata_t *u, const lcsdata_t *v, const lcsdata_t *w, lcsdata_t time, bool device_ptrs,
                    std::string &msg) override {
    if (begun_) {
      msg = "update: previous update not finished";
      return false;
    }
    if (n[0] != n_[0] || n[1] != n_[1] || n[2] != n_[2]) {
      msg = "update: received velocity array of incorrect dimension";
      return false;
    }
    if (first_call_) {
      t_n_ = time;
      t_np1_ = time;
      first_call_ = false;
    } else {
      t_n_ = t_np1_;
      t_np1_ = time;
    }
    cur_ ^= 1;  // u_n = u_np1 (buffer swap); u_np1 is rewritten below
    const int raw_interp = opt_->interpolator;
    if (raw_interp != NEAREST_NBR && raw_interp != LINEAR && raw_interp != QUADRATIC && raw_interp != CUBIC && raw_interp != TSE &&
        raw_interp != TSE_LIMIT) {
      msg = "ERROR: Unrecognized interpolator";
      return false;
    }
    const int interp = interpolator();
    // --- K0 ingest --------------------------------------------------------------------
    CK(cudaEventRecord(ev_[8], stream_));
    CK(cudaEventRecord(ev_[0], stream_));
    const lcsdata_t *su = u, *sv = v, *sw = w;
    if (!device_ptrs) {
      CK(cudaMemcpyAsync(stage_, u, N_ * sizeof(lcsdata_t), cudaMemcpyHostToDevice, stream_));
      CK(cudaMemcpyAsync(stage_ + N_, v, N_ * sizeof(lcsdata_t), cudaMemcpyHostToDevice, stream_));
      CK(cudaMemcpyAsync(stage_ + 2 * N_, w, N_ * sizeof(lcsdata_t), cudaMemcpyHostToDevice, stream_));
      su = stage_;
      sv = stage_ + N_;
      sw = stage_ + 2 * N_;
    }
    DevReduce init{};
    init.cmax = 0ull;
    double big = std::numeric_limits<double>::max();
    std::memcpy(&init.cmin, &big, sizeof(double));
    init.err = red_err_;
    *red_host_ = init;
    CK(cudaMemcpyAsync(red_, red_host_, sizeof(DevReduce), cudaMemcpyHostToDevice, stream_));
    {
      const dim3 blk(32, 8, 1), grd((n_[0] + 31) / 32, (n_[1] + 7) / 8, n_[2]);
      TV *const *U = u_[cur_];
      counters_.kernel_launches++;
      if (dg_.P.has_flags)
        k_ingest<T, TV, lcsdata_t, true><<<grd, blk, 0, stream_>>>(dg_, su, sv, sw, U[0], U[1], U[2], red_);
      else
        k_ingest<T, TV, lcsdata_t, false><<<grd, blk, 0, stream_>>>(dg_, su, sv, sw, U[0], U[1], U[2], red_);
      CK(cudaGetLastError());
    }
    const bool spline = interp == QUADRATIC || interp == CUBIC;
    const int deg = interp == QUADRATIC ? 2 : 3;
    if (spline) {
      if (!ensure_spline(deg, msg)) return false;
      for (int l = 0; l < 2; l++)
        if (!ucoef_[l][0])
          for (int c = 0; c < 3; c++)
            if (!(ucoef_[l][c] = arena_.alloc<TV>(ntot_, msg))) return false;
      if (ucoef_deg_[cur_ ^ 1] != deg) {  // coefficients of u_n missing (first spline use)
        if (!fit(vsplines_[deg].axes, u_[cur_ ^ 1], ucoef_[cur_ ^ 1], msg)) return false;
        ucoef_deg_[cur_ ^ 1] = deg;
      }
      if (!fit(vsplines_[deg].axes, u_[cur_], ucoef_[cur_], msg)) return false;
      ucoef_deg_[cur_] = deg;
    } else {
      ucoef_deg_[cur_] = 0;
    }
    CK(cudaMemcpyAsync(red_host_, red_, sizeof(DevReduce), cudaMemcpyDeviceToHost, stream_));
    CK(cudaEventRecord(ev_[1], stream_));
    begun_ = true;
    return true;
  }

  // Second part: waits for the CFL maximum only, then enqueues every diagnostic's subcycles
  // and the h-boundary work without further host waits (timings are read in update_collect).
  // The batched form runs update_begin for all its instances, then update_enqueue for all,
  // then update_collect, so the instances' kernels overlap on the device.
  bool update_enqueue(std::string &msg) override {
    if (!begun_) {
      msg = "update: no update begun";
      return false;
    }
    begun_ = false;
    evnext_ = 0;
    spans_.clear();
    const int interp = interpolator();
    const bool spline = interp == QUADRATIC || interp == CUBIC;
    const int deg = interp == QUADRATIC ? 2 : 3;
    CK(cudaEventSynchronize(ev_[1]));
    red_err_ = red_host_->err;
    if (red_err_) return err_msg(msg);
    double cmax, cmin;
    std::memcpy(&cmax, &red_host_->cmax, sizeof(double));
    std::memcpy(&cmin, &red_host_->cmin, sizeof(double));
    const lcsdata_t dt_f = t_np1_ - t_n_;
    const lcsdata_t this_cfl = dt_f >= lcsdata_t(0) ? (lcsdata_t)cmax * dt_f : (lcsdata_t)cmin * dt_f;
    counters_.updates++;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    counters_.phase_ms[0] += ms;

    VelFields<TV> V{};
    for (int c = 0; c < 3; c++) {
      V.un[c] = u_[cur_ ^ 1][c];
      V.unp1[c] = u_[cur_][c];
    }
    const SplineAxes<T> sa = spline ? splines_[deg].axes : SplineAxes<T>{};
    const int iv = interp_variant(interp, sa);

    if (spline)
      for (auto &d : diags_) {
        if (d.lg && !ensure_lcs_spline(*d.lg, deg, msg)) return false;
        // every spline buffer of the set at its first spline update, so that later updates
        // (the frames that compose each ring slot for the first time) allocate nothing
        if (d.type == LP_TRACER) continue;
        if (d.type == FTLE_BKWD && !d.fmcoef[0])
          for (int c = 0; c < 3; c++)
            if (!(d.fmcoef[c] = arena_.alloc<T>(dT(d), msg))) return false;
        for (int q = 0; q < d.nslot; q++)
          if (!d.slotcoef[3 * q])
            for (int c = 0; c < 3; c++)
              if (!(d.slotcoef[3 * q + c] = arena_.alloc<T>(dT(d), msg))) return false;
      }
    // --- per particle set: K1 (backward) / K6 (forward) --------------------------------
    for (auto &d : diags_) {
      if (!d.active) continue;
      // stage blends belong to one particle set: a set that samples the levels per corner must
      // not see the blends (other stage times) the previous set left in V
      for (auto &row : V.cs)
        for (auto &ptr : row) ptr = nullptr;
      const lcsdata_t q = this_cfl / (lcsdata_t(opt_->cfl) * d.dt_factor);
      long nsub = (long)std::ceil((double)q);
      if (!(q == q)) {
        msg = "set_dt: non-finite CFL number";
        return false;
      }
      if (nsub < 1) nsub = 1;
      lcsdata_t dt = dt_f / (lcsdata_t)nsub;
      if (d.type == FTLE_BKWD) dt = lcsdata_t(-1) * dt;
      const long long npart = d.type == LP_TRACER ? (long long)d.np : (long long)dN(d);
      if (std::fabs((double)dt) > 0) {
        if (d.type != FTLE_BKWD) counters_.integrations_fwd += npart * nsub;
        else counters_.integrations_bkwd += npart * nsub;
      }
      if (d.type != FTLE_BKWD) counters_.nsub_fwd = nsub;
      else counters_.nsub_bkwd = nsub;
      cudaEvent_t adv0, adv1;
      if (!mark(adv0, msg)) return false;
      lcsdata_t lp_time = d.type == FTLE_BKWD ? t_np1_ : t_n_;
      const int kkind = d.type == FTLE_BKWD ? SPAN_SL : SPAN_FWD;
      for (long sc = 0; sc < nsub; sc++) {
        cudaEvent_t k0, k1;
        StageTimes S = stage_times(lp_time, dt);
        if ((spline || (interp == LINEAR && N_ >= lin_blend_min_ && (d.type != FTLE_BKWD || d.lg))) && !stage_blends(d, S, V, msg))
          return false;
        if (d.type == FTLE_BKWD) {
          FieldPtrs<T> fo;
          FieldPtrsW<T> fn;
          for (int c = 0; c < 3; c++) {
            fo.f[c] = d.fm[d.cur][c];
            fn.f[c] = d.fm[d.cur ^ 1][c];
          }
          if (spline) {
            if (!d.fmcoef[0])
              for (int c = 0; c < 3; c++)
                if (!(d.fmcoef[c] = arena_.alloc<T>(dT(d), msg))) return false;
            if (!fit(d.lg ? d.lg->sp[deg].axes : splines_[deg].axes, d.fm[d.cur], d.fmcoef, msg, &dgrid(d))) return false;
            for (int c = 0; c < 3; c++) fo.f[c] = d.fmcoef[c];
          }
          if (!mark(k0, msg)) return false;
          if (d.lg ? !launch_sl_refined(d, sa, spline ? d.lg->sp[deg].axes : SplineAxes<T>{}, V, fo, fn, S, (T)dt, msg)
                   : !launch_sl(iv, sa, V, fo, fn, S, (T)dt, msg))
            return false;
          if (!mark(k1, msg)) return false;
          spans_.push_back({k0, k1, kkind, !d.lg && sl_variant_ >= 0 && tune_[0].choice < 0 && tile_mode_ == 1 ? sl_variant_ : -1});
          d.cur ^= 1;
        } else if (d.type == LP_TRACER) {
          // tracers: the forward subcycle on their own particles (few, unsorted)
          if (!launch_fwd(iv, sa, V, d.P, S, (T)dt, msg, d.np)) return false;
          d.lifetime = d.lifetime + (lcsdata_t)std::fabs((double)dt);  // integrate_lp, lp_motion_m.f90:332
        } else {
          // the variant holds from one sort to the next (the staged kernel reads the sort's tiles)
          const bool usable = fwd_tile_usable(iv, V);
          // the staged family re-sorts every kSortInterval subcycles of the update (its tiles
          // must be the sort's); the gathering-only sets re-sort when their launches have lost
          // more time to disorder than a sort costs (sort_due)
          const int di = (int)(&d - diags_.data());
          const bool resort = usable ? sc % sort_interval(interp) == 0 : sort_due(d);
          if (resort) {
            d.fwd_variant = usable ? tile_variant(1) : 0;
            cudaEvent_t s0, s1;
            if (!usable && !mark(s0, msg)) return false;
            if (!sort_particles(d, msg, d.fwd_variant == 1)) return false;
            if (!usable) {
              if (!mark(s1, msg)) return false;
              spans_.push_back({s0, s1, SPAN_SORT, -1, di, 0});
            }
            d.since_sort = 0;
            d.excess_ms = 0;
          }
          const bool staged = usable && d.fwd_variant == 1;
          if (!mark(k0, msg)) return false;
          if (staged ? !launch_fwd_tile(d, sa, V, S, (T)dt, msg) : !launch_fwd(iv, sa, V, d.P, S, (T)dt, msg, dN(d))) return false;
          if (!mark(k1, msg)) return false;
          spans_.push_back({k0, k1, kkind, usable && tune_[1].choice < 0 && tile_mode_ == 1 ? 2 + d.fwd_variant : -1, usable ? -1 : di,
                            (int)std::min(d.since_sort, 1L << 30)});
          d.since_sort++;
        }
        lp_time = lp_time + dt;
      }
      if (!mark(adv1, msg)) return false;
      spans_.push_back({adv0, adv1, d.type == FTLE_BKWD ? 1 : 2});
    }

    // --- h boundaries: K7 snapshot, K4 composition, K5 FTLE, reset ----------------------
    // (auxiliary sets first: a diagnostic's AUX_GRID FTLE reads their composed maps)
    for (int pass = 0; pass < 2; pass++)
    for (auto &d : diags_) {
      if ((d.aux_parent != 0) != (pass == 0)) continue;
      if (!d.active) continue;
      if ((long)(t_np1_ / d.h) == (long)(t_n_ / d.h)) continue;
      if (d.type == LP_TRACER) {
        // write_lcs, then the end of the tracers' lifetime (src/cfd2lcs.f90:225-231)
        if (opt_->write_lcs && !enqueue_tracer_output(d, msg)) return false;
        if (d.lifetime > d.T_) d.active = false;
        continue;
      }
      cudaEvent_t f4, f5, f6, f7;
      if (!mark(f4, msg)) return false;
      const long step0 = fnint((double)(lcsdata_t)std::fmod((double)t_np1_, (double)d.T_) / (double)d.h);
      // the reference writes slot nint(mod(t,T)/h); slot nint(T/h) and negative slots go to
      // files reconstruct never reads back
      const long wslot = fnint((double)((lcsdata_t)std::fmod((double)t_np1_, (double)d.T_) / d.h));
      (void)step0;
      if (need_velocity_ring() && !snapshot_velocity(wslot, msg)) return false;
      if (wslot >= 0 && wslot < d.nslot) {
        if (!launch_snapshot(d, (int)wslot, msg)) return false;
        d.written[wslot] = 1;
        d.coef_deg[wslot] = 0;
      }
      if (!mark(f5, msg)) return false;
      // composition order (reconstruct_flowmap, src/flowmap_m.f90:202-268)
      const int nstep = d.nslot;
      long step = wslot;
      const int inc = d.type == FTLE_FWD ? 1 : -1;
      if (d.type == FTLE_FWD) step += inc;
      int m = 0;
      d.last_order.clear();
      for (int i = 0; i < nstep; i++) {
        if (step >= nstep) step = 0;
        if (step < 0) step = nstep - 1;
        if (d.written[step]) {
          if (spline) {
            if (!d.slotcoef[3 * step])
              for (int c = 0; c < 3; c++)
                if (!(d.slotcoef[3 * step + c] = arena_.alloc<T>(dT(d), msg))) return false;
            if (d.coef_deg[step] != deg) {
              if (!fit(d.lg ? d.lg->sp[deg].axes : splines_[deg].axes, &d.slot[3 * step], &d.slotcoef[3 * step], msg, &dgrid(d)))
                return false;
              d.coef_deg[step] = deg;
            }
            for (int c = 0; c < 3; c++) d.slot_list_host[3 * m + c] = d.slotcoef[3 * step + c];
          } else {
            for (int c = 0; c < 3; c++) d.slot_list_host[3 * m + c] = d.slot[3 * step + c];
          }
          d.last_order.push_back((int)step);
          m++;
        }
        step += inc;
      }
      CK(cudaMemcpyAsync(d.slot_list_dev, d.slot_list_host.data(), sizeof(T *) * 3 * std::max(m, 1), cudaMemcpyHostToDevice,
                         stream_));
      if (d.lg && spline) {
        const SplineAxes<T> &la = d.lg->sp[deg].axes;
        if (!launch_compose(interp_variant(interp, la), la, d, m, msg)) return false;
      } else if (!launch_compose(iv, sa, d, m, msg)) {
        return false;
      }
      if (!mark(f6, msg)) return false;
      if (!d.aux_parent) {
        if (opt_->aux_grid && d.aux.empty()) {
          msg = "AUX_GRID was set after cfd2lcs_diagnostic_init: this diagnostic has no auxiliary particle sets";
          return false;
        }
        if (d.aux.empty() ? !launch_ftle(d, msg) : !launch_ftle_aux(d, msg)) return false;
        // lp%ugrid of a refined lcs grid, read by the invariants and the output file
        if (d.lg && need_velocity_ring() && !make_ugrid(d, wslot + (d.type == FTLE_FWD ? 1 : 0), msg)) return false;
        // compute_invariants from the velocity of the reconstruction's starting step: the
        // current one (backward) or the next, not yet wrapped (forward), flowmap_m.f90:202-245
        if (opt_->velocity_invariants && !launch_invariants(d, wslot + (d.type == FTLE_FWD ? 1 : 0), msg)) return false;
        // write_lcs (src/cfd2lcs.f90:202): the frame's file, staged now, written by the writer
        if (opt_->write_lcs && !enqueue_output(d, wslot + (d.type == FTLE_FWD ? 1 : 0), msg)) return false;
      }
      if (!mark(f7, msg)) return false;
      // reset_lp: particles back to the grid, flow map to zero (src/cfd2lcs.f90:208-209)
      if (d.type == FTLE_BKWD) {
        for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(d.fm[d.cur][c], 0, dT(d) * sizeof(T), stream_));
        if (d.lg && !reset_refined_nodes(d, msg)) return false;
      } else {
        launch_reset(d);
      }
      // (the slot pointer list was copied from pageable host memory: cudaMemcpyAsync returns
      // once the source is staged, so the host vector may be rewritten by the next frame)
      spans_.push_back({f4, f5, 3});
      spans_.push_back({f5, f6, 4});
      spans_.push_back({f6, f7, 5});
      d.have_frame = true;
      if (!d.aux_parent) counters_.ftle_frames++;
    }
    CK(cudaEventRecord(ev_[9], stream_));
    return true;
  }

  // Last part: waits for the update's final event, accumulates the event-timed phases and
  // kernels, and folds the device error word into the result.
  bool update_collect(std::string &msg) override {
    CK(cudaEventSynchronize(ev_[9]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_[8], ev_[9]));
    counters_.phase_ms[6] += ms;
    for (const Span &sp : spans_) {
      CK(cudaEventElapsedTime(&ms, sp.a, sp.b));
      if (sp.tune >= 0) tune_record(sp.tune, ms);
      if (sp.kind == SPAN_SL) {
        counters_.sl_kernel_ms += ms;
        counters_.sl_kernel_launches++;
      } else if (sp.kind == SPAN_FWD) {
        counters_.fwd_kernel_ms += ms;
        counters_.fwd_kernel_launches++;
        if (sp.diag >= 0 && sp.diag < (int)diags_.size()) {
          DiagT &d = diags_[sp.diag];
          if (sp.since == 0 || d.base_ms < 0) d.base_ms = ms;
          else d.excess_ms += std::max(0.0, (double)ms - d.base_ms);
        }
      } else if (sp.kind == SPAN_SORT) {
        if (sp.diag >= 0 && sp.diag < (int)diags_.size()) {
          diags_[sp.diag].sort_ms = ms;
          diags_[sp.diag].excess_ms = 0;  // launches collected before it belong to the old order
        }
      } else {
        counters_.phase_ms[sp.kind] += ms;
      }
    }
    spans_.clear();
    if (writer_) {
      if (!opt_->write_lcs_async) writer_->flush();  // the reference's file is complete on return
      const std::string e = writer_->take_error();
      if (!e.empty()) {
        msg = e;
        return false;
      }
    }
    return sync_errors(msg);
  }

  bool sync_errors(std::string &msg) override {
    if (!stream_) return true;
    CK(cudaStreamSynchronize(stream_));
    int err = 0;
    CK(cudaMemcpy(&err, &red_->err, sizeof(int), cudaMemcpyDeviceToHost));
    red_err_ |= err;
    if (red_err_) return err_msg(msg);
    return true;
  }

  bool reconstruct_noalloc(int handle, lcsdata_t *d_ftle, lcsdata_t *d_fm, std::string &msg) override {
    DiagT *d = find(handle);
    if (!d || !d->have_frame) {
      msg = "reconstruct_noalloc: unknown handle or no FTLE frame yet";
      return false;
    }
    if (d->lg || !d->aux.empty()) {
      msg = "reconstruct_noalloc: diagnostics with resolution /= 0 or AUX_GRID are not supported";
      return false;
    }
    const int m = (int)d->last_order.size();
    if (m > NOALLOC_MAX_SUBMAPS) {
      msg = "reconstruct_noalloc: the frame composes " + std::to_string(m) + " sub-flow maps, more than the maximum of " +
            std::to_string(NOALLOC_MAX_SUBMAPS) + " (T/h too large)";
      return false;
    }
    const int interp = interpolator();
    const bool spline = interp == QUADRATIC || interp == CUBIC;
    const int deg = interp == QUADRATIC ? 2 : 3;
    const T *host_table[3 * NOALLOC_MAX_SUBMAPS];
    for (int q = 0; q < m; q++) {
      const int s = d->last_order[q];
      if (spline && (d->coef_deg[s] != deg || !d->slotcoef[3 * s])) {
        msg = "reconstruct_noalloc: the stored sub-flow maps have no spline coefficients for the current interpolator";
        return false;
      }
      for (int c = 0; c < 3; c++) host_table[3 * q + c] = spline ? d->slotcoef[3 * s + c] : d->slot[3 * s + c];
    }
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != dev_) {
      msg = "reconstruct_noalloc: the current CUDA device (" + std::to_string(cur) + ") is not the device cfd2lcs_init ran on (" +
            std::to_string(dev_) + ")";
      return false;
    }
    void *table = nullptr;
    if (!noalloc_table_address(dev_, &table, msg)) return false;
    if (m > 0) CK(cudaMemcpyAsync(table, host_table, sizeof(T *) * 3 * m, cudaMemcpyHostToDevice, stream_));
    const SplineAxes<T> sa = spline ? splines_[deg].axes : SplineAxes<T>{};
    const int iv = interp_variant(interp, sa);
    FieldPtrsW<T> out{};
    for (int c = 0; c < 3; c++) out.f[c] = reinterpret_cast<T *>(d_fm) + (size_t)c * N_;
    const dim3 blk(32, 8, 1), grd = node_grid();
    int *err = &red_->err;
    const bool F = dg_.P.has_flags != 0;
    const T *const *sl = reinterpret_cast<const T *const *>(table);
#define COMPOSE_NA(I, FL) k_compose<T, I, FL><<<grd, blk, 0, stream_>>>(dg_, sa, sl, m, out, err)
    if (iv == INTERP_NEAREST) { if (F) COMPOSE_NA(INTERP_NEAREST, true); else COMPOSE_NA(INTERP_NEAREST, false); }
    else if (iv == INTERP_LINEAR) { if (F) COMPOSE_NA(INTERP_LINEAR, true); else COMPOSE_NA(INTERP_LINEAR, false); }
    else if (iv == INTERP_TSE) { if (F) COMPOSE_NA(INTERP_TSE, true); else COMPOSE_NA(INTERP_TSE, false); }
    else if (iv == INTERP_TSE_LIMIT) { if (F) COMPOSE_NA(INTERP_TSE_LIMIT, true); else COMPOSE_NA(INTERP_TSE_LIMIT, false); }
    else if (iv == INTERP_CTSE) { if (F) COMPOSE_NA(INTERP_CTSE, true); else COMPOSE_NA(INTERP_CTSE, false); }
    else if (iv == INTERP_CTSE_LIMIT) { if (F) COMPOSE_NA(INTERP_CTSE_LIMIT, true); else COMPOSE_NA(INTERP_CTSE_LIMIT, false); }
    else if (iv == INTERP_SPLINE4) { if (F) COMPOSE_NA(INTERP_SPLINE4, true); else COMPOSE_NA(INTERP_SPLINE4, false); }
    else { if (F) COMPOSE_NA(INTERP_SPLINE, true); else COMPOSE_NA(INTERP_SPLINE, false); }
#undef COMPOSE_NA
    CK(cudaGetLastError());
    FieldPtrs<T> f{};
    for (int c = 0; c < 3; c++) f.f[c] = out.f[c];
    launch_ftle(dg_, f, d_ftle, d->T_, blk, grd);
    CK(cudaGetLastError());
    return sync_errors(msg);
  }

  bool get_ftle(int handle, lcsdata_t *out, std::string &msg) override {
    DiagT *d = find(handle);
    if (!d || !d->have_frame) {
      msg = "get_ftle: unknown handle or no FTLE frame yet";
      return false;
    }
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(out, d->ftle, dN(*d) * sizeof(lcsdata_t), cudaMemcpyDeviceToHost));
    return true;
  }

  bool get_flowmap(int handle, lcsdata_t *out, std::string &msg) override {
    DiagT *d = find(handle);
    if (!d || !d->have_frame) {
      msg = "get_flowmap: unknown handle or no FTLE frame yet";
      return false;
    }
    CK(cudaStreamSynchronize(stream_));
    const long nd = dN(*d);
    std::vector<T> tmp(nd);
    for (int c = 0; c < 3; c++) {
      CK(cudaMemcpy(tmp.data(), d->composed[c], nd * sizeof(T), cudaMemcpyDeviceToHost));
      for (long q = 0; q < nd; q++) out[c * nd + q] = (lcsdata_t)tmp[q];
    }
    return true;
  }

  bool get_invariants(int handle, lcsdata_t *out, std::string &msg) override {
    DiagT *d = find(handle);
    if (!d || !d->have_frame || !d->inv[0]) {
      msg = "get_invariants: unknown handle, no frame yet, or VELOCITY_INVARIANTS off";
      return false;
    }
    CK(cudaStreamSynchronize(stream_));
    const long nd = dN(*d);
    for (int q = 0; q < 5; q++) CK(cudaMemcpy(out + (size_t)q * nd, d->inv[q], nd * sizeof(lcsdata_t), cudaMemcpyDeviceToHost));
    return true;
  }

  bool diagnostic_size(int handle, int n[3]) override {
    DiagT *d = find(handle);
    if (!d) return false;
    for (int a = 0; a < 3; a++) n[a] = d->lg ? d->lg->dg.P.n[a] : n_[a];
    return true;
  }

  int tracer_count(int handle) override {
    DiagT *d = find(handle);
    return d && d->type == LP_TRACER ? d->np : -1;
  }

  // positions of a tracer set (the last ones it reached: after its lifetime the reference
  // destroys the set, here it stops moving)
  bool get_tracers(int handle, lcsdata_t *out, std::string &msg) override {
    DiagT *d = find(handle);
    if (!d || d->type != LP_TRACER) {
      msg = "get_tracers: not an LP_TRACER handle";
      return false;
    }
    CK(cudaStreamSynchronize(stream_));
    std::vector<T> tmp(d->np);
    for (int c = 0; c < 3; c++) {
      if (d->np) CK(cudaMemcpy(tmp.data(), d->P.x[c], d->np * sizeof(T), cudaMemcpyDeviceToHost));
      for (int q = 0; q < d->np; q++) out[(size_t)c * d->np + q] = (lcsdata_t)tmp[q];
    }
    return true;
  }

  const lcsdata_t *ftle_device_ptr(int handle) override {
    DiagT *d = find(handle);
    return d ? d->ftle : nullptr;
  }

  const Counters &counters() const override { return counters_; }

 private:
  int fail(std::string &msg, const char *what) {
    msg = std::string("CUDA error in ") + what;
    return -1;
  }

  // LP_TRACER (init_lp_tracer, src/lp_m.f90:116-226, and diagnostic_init, src/cfd2lcs.f90:
  // 327-337): one particle per grid node inside the injection sphere, r <= radius, in node
  // order (i fastest), starting at the node (where node tracking leaves it).  With no node
  // inside, the set is dropped and the handle is -1 (-2 here: not an error); its number is
  // used up all the same, as the reference's diagnostic count is.
  int tracer_init(lcsdata_t Tint, lcsdata_t h, const char *label, int resolution, std::string &msg) {
    if (!(h > lcsdata_t(0)) || !(Tint > lcsdata_t(0))) {
      msg = "diagnostic_init: T and h must be positive";
      return -1;
    }
    DiagT d;
    d.handle = ++handle_count_;
    d.type = LP_TRACER;
    d.T_ = Tint;
    d.h = h;
    d.dt_factor = lcsdata_t(1);
    d.label = label ? label : "";
    while (!d.label.empty() && d.label.back() == ' ') d.label.pop_back();
    const lcsdata_t X = (lcsdata_t)opt_->tracer_x, Y = (lcsdata_t)opt_->tracer_y, Z = (lcsdata_t)opt_->tracer_z;
    const lcsdata_t R = (lcsdata_t)opt_->tracer_r;
    std::vector<T> px[3];
    std::vector<int> pn[3];
    // on a refined lcs grid (resolution /= 0) the injected nodes are that grid's, tracked to
    // the solver grid with the periodic wrap (track_lp2node of init_lp_tracer's set)
    DiagT tmp;
    if (resolution != 0 && !make_lcs_grid(tmp, FTLE_FWD, resolution, msg)) return -1;
    const HostGrid<lcsdata_t> &G = tmp.lg ? tmp.lg->hg : hg_;
    std::vector<T> tpos[3];
    std::vector<int> tnos[3];
    if (tmp.lg) {
      if (cudaStreamSynchronize(stream_) != cudaSuccess) return fail(msg, "sync");
      for (int c = 0; c < 3; c++) {
        tpos[c].resize(tmp.lg->N);
        tnos[c].resize(tmp.lg->N);
        if (cudaMemcpy(tpos[c].data(), tmp.lg->pos[c], tmp.lg->N * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(tnos[c].data(), tmp.lg->nos_reset[c], tmp.lg->N * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
          return fail(msg, "tracer node copy");
      }
    }
    long q = 0;
    for (int k = 1; k <= G.P.n[2]; k++)
      for (int j = 1; j <= G.P.n[1]; j++)
        for (int i = 1; i <= G.P.n[0]; i++, q++) {
          const lcsdata_t dx = G.coord(0, i, j, k) - X, dy = G.coord(1, i, j, k) - Y, dz = G.coord(2, i, j, k) - Z;
          const lcsdata_t r = std::sqrt(dx * dx + dy * dy + dz * dz);
          if (!(r <= R)) continue;
          const int nd[3] = {i, j, k};
          for (int a = 0; a < 3; a++) {
            px[a].push_back(tmp.lg ? tpos[a][q] : (T)G.coord(a, i, j, k));
            pn[a].push_back(tmp.lg ? tnos[a][q] : nd[a]);
          }
        }
    d.np = (int)px[0].size();
    if (d.np == 0) {
      d.active = false;
      diags_.push_back(std::move(d));
      return -2;
    }
    std::vector<T> zero(d.np, T(0));
    for (int c = 0; c < 3; c++) {
      if (!(d.P.x[c] = upload<T>(px[c], msg))) return -1;
      if (!(d.P.dx[c] = upload<T>(zero, msg))) return -1;
      if (!(d.P.no[c] = upload<int>(pn[c], msg))) return -1;
    }
    diags_.push_back(std::move(d));
    return diags_.back().handle;
  }

  // write_tracers (src/io_nohdf5_m.f90:138-181): POINT-packed positions, one particle per line
  bool enqueue_tracer_output(DiagT &d, std::string &msg) {
    const long long findex = (long long)fnint((double)(t_np1_ / d.h));
    std::string idx;
    if (!lcs_file_index(findex, idx)) {
      msg = "ERROR: unsupported range for file index, " + std::to_string(findex);
      return false;
    }
    if (!writer_) writer_.reset(new LcsWriter());
    OutputJob job;
    job.path = "./cfd2lcs_output/" + d.label + "_" + idx + ".dat";
    job.points = d.np;
    const std::string lab = d.label + "-LP";
    std::string h = "TITLE = \"" + lab + "\"\nVARIABLES =\n\"X\"\n\"Y\"\n\"Z\"\nZONE\nT = \"" + lab + "\"\n";
    char tbuf[32], line[160];
    format_es((double)t_np1_, 18, 4, tbuf);
    tbuf[18] = 0;
    std::snprintf(line, sizeof(line), "STRANDID = %010d, SOLUTIONTIME = %s\n", d.handle + 1, tbuf);
    h += line;
    std::snprintf(line, sizeof(line), "I = %010d J = %010d K = %010d\n", d.np, 1, 1);
    h += line;
    h += "ZONETYPE = Ordered, DATAPACKING = POINT\n";
    job.header = h;
    const size_t blk = ((size_t)d.np * sizeof(T) + 255) / 256 * 256;
    void *buf = nullptr;
    const int bi = writer_->acquire(std::max<size_t>(3 * blk, 1), &buf, msg);
    if (bi < 0) return false;
    for (int c = 0; c < 3; c++) {
      OutputBlock b;
      b.kind = sizeof(T) == 8 ? OutputBlock::STAGED_F64 : OutputBlock::STAGED_F32;
      b.offset = c * blk;
      job.blocks.push_back(b);
      if (d.np) CK(cudaMemcpyAsync(static_cast<char *>(buf) + b.offset, d.P.x[c], d.np * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    }
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, stream_));
    job.ready = ev;
    job.buffer = bi;
    writer_->submit(std::move(job));
    return true;
  }

  bool err_msg(std::string &msg) {
    if (red_err_ & ERR_NONFINITE_VELOCITY) msg = "update: non-finite velocity (CFL number is not finite)";
    else if (red_err_ & ERR_TRACKING) msg = "ERROR: cannot locate all particles (node search did not converge)";
    else if (red_err_ & ERR_UNKNOWN_FLAG) msg = "ERROR: Unknown bcflag";
    else if (red_err_ & ERR_ASYNC_COPY) msg = "device error: a shared-memory staging copy did not complete";
    else msg = "device error";
    return false;
  }

  template <typename D = T, typename V>
  D *upload(const std::vector<V> &h, std::string &msg) {
    std::vector<D> tmp(h.size());
    for (size_t q = 0; q < h.size(); q++) tmp[q] = (D)h[q];
    D *d = arena_.alloc<D>(tmp.size(), msg);
    if (!d) return nullptr;
    if (cudaMemcpy(d, tmp.data(), tmp.size() * sizeof(D), cudaMemcpyHostToDevice) != cudaSuccess) {
      msg = "upload failed";
      return nullptr;
    }
    return d;
  }

  DiagT *find(int handle) {
    for (auto &d : diags_)
      if (d.handle == handle) return &d;
    return nullptr;
  }

  // stage time fractions of integrate_lp (src/lp_motion_m.f90:165-327) in the interface
  // precision, as the reference computes them
  StageTimes stage_times(lcsdata_t t, lcsdata_t dt) const {
    const lcsdata_t t0 = t_n_, t1 = t_np1_;
    const lcsdata_t HALF = lcsdata_t(1) / lcsdata_t(2);
    auto ct = [&](lcsdata_t tt) -> double {
      if (t1 == t0) return 0.0;  // first update: 0/0, the displacement is zero for any ct
      lcsdata_t v = (tt - t0) / (t1 - t0);
      v = std::max(std::min(v, lcsdata_t(1)), lcsdata_t(0));
      return (double)v;
    };
    StageTimes S{};
    switch (opt_->integrator) {
      case 0: S.ct[0] = ct(t); break;
      case 1: S.ct[0] = ct(t + HALF * dt); break;
      case 2: S.ct[0] = ct(t); S.ct[1] = ct(t + HALF * dt); break;
      case 3: S.ct[0] = ct(t); S.ct[1] = ct(t + HALF * dt); S.ct[2] = ct(t + dt); break;
      default: S.ct[0] = ct(t); S.ct[1] = ct(t + HALF * dt); S.ct[2] = S.ct[1]; S.ct[3] = ct(t + dt); break;
    }
    return S;
  }

  // Coefficients of the blended stage velocities of one subcycle, in the diagnostic's three
  // blend buffers.  A buffer already holding the same ct of this update is reused (the last
  // stage of a subcycle is the first of the next; RK4's two midpoint stages coincide).
  bool stage_blends(DiagT &d, const StageTimes &S, VelFields<TV> &V, std::string &msg) {
    static const int nst[5] = {1, 1, 2, 3, 4};
    const int ns = nst[std::min(std::max(opt_->integrator, 0), 4)];
    const long long upd = counters_.updates;
    bool used[3] = {false, false, false};
    int pick[4] = {-1, -1, -1, -1};
    for (int st = 0; st < ns; st++)
      for (int b = 0; b < 3; b++)
        if (d.blend[b][0] && d.blend_update[b] == upd && d.blend_ct[b] == S.ct[st]) {
          pick[st] = b;
          used[b] = true;
          break;
        }
    BlendOut<TV> o{};
    int nout = 0;
    for (int st = 0; st < ns; st++) {
      if (pick[st] >= 0) continue;
      for (int q = 0; q < st; q++)
        if (S.ct[q] == S.ct[st] && pick[q] >= 0) pick[st] = pick[q];
      if (pick[st] >= 0) continue;
      int b = 0;
      while (b < 3 && used[b]) b++;
      if (b == 3) {
        msg = "internal: no free blend buffer";
        return false;
      }
      if (!d.blend[b][0])
        for (int c = 0; c < 3; c++)
          if (!(d.blend[b][c] = arena_.alloc<TV>(ntot_, msg))) return false;
      const TV ct = (TV)S.ct[st];
      for (int c = 0; c < 3; c++) o.f[nout][c] = d.blend[b][c];
      o.omc[nout] = TV(1) - ct;
      o.ct[nout] = ct;
      nout++;
      d.blend_ct[b] = S.ct[st];
      d.blend_update[b] = upd;
      used[b] = true;
      pick[st] = b;
    }
    if (nout > 0) {
      FieldPtrs<TV> a{}, bb{};
      // B-splines blend the levels' coefficients, LINEAR the levels themselves
      const bool spl = opt_->interpolator == QUADRATIC || opt_->interpolator == CUBIC;
      for (int c = 0; c < 3; c++) {
        a.f[c] = spl ? ucoef_[cur_ ^ 1][c] : u_[cur_ ^ 1][c];
        bb.f[c] = spl ? ucoef_[cur_][c] : u_[cur_][c];
      }
      const long npair = (ntot_ + 1) / 2;
      const dim3 grd((unsigned)((npair + 255) / 256), 3);
      k_blend<TV><<<grd, 256, 0, stream_>>>(a, bb, o, nout, ntot_);
      counters_.kernel_launches++;
      CK(cudaGetLastError());
    }
    for (int st = 0; st < ns; st++)
      for (int c = 0; c < 3; c++) V.cs[st][c] = d.blend[pick[st]][c];
    return true;
  }

  // LINEAR interpolation writes each stage's time blend once per subcycle (k_blend) for the
  // particle sets whose every stage is off the nodes (forward particles, refined backward sets)
  // on grids of at least this many points, so that every particle gathers 8 blended corners
  // instead of 8 x 2 levels.  Measured on B200: the forward kernel 1.64 -> 1.17 ms per launch on
  // ABC 256^3 RK2; the backward SL kernel, whose first stage reads the nodal values, gained less
  // than the blend pass cost (turbulence 512^3: 140 -> 155 ms per update), so it keeps the
  // per-corner blend; on small grids the extra pass costs more than it saves.  The environment
  // variable CFD2LCS_B200_LINEAR_BLEND_MIN, read at cfd2lcs_init, overrides it (the tests take
  // the blended path on small grids with it).
#ifndef CFD2LCS_LINEAR_BLEND_MIN
#define CFD2LCS_LINEAR_BLEND_MIN (1L << 22)
#endif
  long lin_blend_min_ = CFD2LCS_LINEAR_BLEND_MIN;

  // B-spline axes (flow-map type) of an lcs grid, as ensure_spline builds the solver grid's
  bool ensure_lcs_spline(LcsGrid<T> &L, int deg, std::string &msg) {
    if (L.sp[deg].deg == deg) return true;
    SplineSet<T> s;
    s.deg = deg;
    for (int a = 0; a < 3; a++) {
      SplineAxisHost<lcsdata_t> A;
      const int npts = L.dg.P.n[a] + 2;
      const int k = std::max(std::min(deg + 1, npts - 1), 2);
      if (!A.build(L.hg.li[a], k)) {
        msg = "bspline: singular collocation system or bad abscissae";
        return false;
      }
      SplineAxis<T> &D = s.axes.ax[a];
      D.n = A.n;
      D.k = A.k;
      if (!(D.t = upload(A.t, msg))) return false;
      if (!(D.rinv = upload(A.rinv, msg))) return false;
      if (!(D.tu = upload(A.tu, msg))) return false;
      if (!(D.pull = upload(pull_table(A), msg))) return false;
    }
    L.sp[deg] = s;
    return true;
  }

  bool ensure_spline(int deg, std::string &msg) {
    if (splines_[deg].deg == deg) return true;
    SplineSet<T> s;
    SplineSet<TV> sv;
    s.deg = sv.deg = deg;
    for (int a = 0; a < 3; a++) {
      SplineAxisHost<lcsdata_t> A;
      const int npts = n_[a] + 2;
      const int k = std::max(std::min(deg + 1, npts - 1), 2);
      if (!A.build(hg_.li[a], k)) {
        msg = "bspline: singular collocation system or bad abscissae";
        return false;
      }
      SplineAxis<T> &D = s.axes.ax[a];
      D.n = A.n;
      D.k = A.k;
      if (!(D.t = upload(A.t, msg))) return false;
      if (!(D.rinv = upload(A.rinv, msg))) return false;
      if (!(D.tu = upload(A.tu, msg))) return false;
      const std::vector<lcsdata_t> pull = pull_table(A);
      if (!(D.pull = upload(pull, msg))) return false;
      // the velocity fits solve with the LU factors rounded to the velocity type
      SplineAxis<TV> &E = sv.axes.ax[a];
      E.n = A.n;
      E.k = A.k;
      if (!(E.t = upload<TV>(A.t, msg))) return false;
      if (!(E.rinv = upload<TV>(A.rinv, msg))) return false;
      if (!(E.tu = upload<TV>(A.tu, msg))) return false;
      if (!(E.pull = upload<TV>(pull, msg))) return false;
    }
    splines_[deg] = s;
    vsplines_[deg] = sv;
    return true;
  }

  static std::vector<lcsdata_t> pull_table(const SplineAxisHost<lcsdata_t> &A) { return spline_pull_table(A); }

  template <typename D, int K>
  void fit_pass(const SplineAxis<D> &A, FieldPtrs<D> s, FieldPtrsW<D> d, int axis, const DevGrid<T> &g) {
    const int sx = g.P.sx, sxy = g.P.sxy, ny = g.P.n[1] + 2, nz = g.P.n[2] + 2;
    if (axis == 0) {
      const long warps = (long)((ny + 31) / 32) * nz;
      const size_t smem = sizeof(D) * 4 * 2 * 32 * (XFIT_W + 1);  // two 32 x (XFIT_W + 1) tiles per warp
      static bool attr_done = false;
      if (!attr_done) {
        cudaFuncSetAttribute(k_fit_xlines<D, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_done = true;
      }
      k_fit_xlines<D, K><<<dim3((unsigned)((warps + 3) / 4), 3), 128, smem, stream_>>>(A, s, d, ny, nz, (long)sx, (long)sxy);
    } else {
      // y lines: sx * nz of them, elements sx apart; z lines: sxy of them, elements sxy apart
      const int nfast = axis == 1 ? sx : sxy;
      const long nlines = axis == 1 ? (long)sx * nz : (long)sxy;
      const long es = axis == 1 ? (long)sx : (long)sxy;
      k_fit_lines<D, K><<<dim3((unsigned)((nlines + 255) / 256), 3), 256, 0, stream_>>>(A, s, d, nfast, nlines, es, (long)sxy);
    }
  }

  template <typename D>
  void fit_pass_any(const SplineAxis<D> &A, FieldPtrs<D> s, FieldPtrsW<D> d, int axis, const DevGrid<T> &g) {
    if (A.k == 4) fit_pass<D, 4>(A, s, d, axis, g);
    else if (A.k == 3) fit_pass<D, 3>(A, s, d, axis, g);
    else fit_pass<D, 2>(A, s, d, axis, g);
  }

  // Coefficients of the padded fields src (3 components) into dst (db3ink: x, then y, then z).
  // D is the field type: T for flow maps and sub-flow maps, TV for velocity levels.
  template <typename D>
  bool fit(const SplineAxes<D> &S, D *const src[3], D *const dst[3], std::string &msg, const DevGrid<T> *grid = nullptr) {
    const DevGrid<T> &g = grid ? *grid : dg_;
    FieldPtrs<D> s{}, di{};
    FieldPtrsW<D> d{};
    for (int c = 0; c < 3; c++) {
      s.f[c] = src[c];
      di.f[c] = dst[c];
      d.f[c] = dst[c];
    }
    counters_.kernel_launches += 3;
    fit_pass_any(S.ax[0], s, d, 0, g);
    fit_pass_any(S.ax[1], di, d, 1, g);
    fit_pass_any(S.ax[2], di, d, 2, g);
    CK(cudaGetLastError());
    return true;
  }

  // The interpolator the kernels run: on a non-rectilinear grid the reference takes TSE_LIMIT
  // unless TSE was asked for (interp_s2u_r1, src/lp_tracking_m.f90:320-327).
  int interpolator() const {
    const int v = opt_->interpolator;
    return hg_.P.curv ? (v == TSE ? TSE : TSE_LIMIT) : v;
  }

  int interp_variant(int interp, const SplineAxes<T> &sa) const {
    if (hg_.P.curv) return interp == TSE ? INTERP_CTSE : INTERP_CTSE_LIMIT;
    if (interp == NEAREST_NBR) return INTERP_NEAREST;
    if (interp == LINEAR) return INTERP_LINEAR;
    if (interp == TSE) return INTERP_TSE;
    if (interp == TSE_LIMIT) return INTERP_TSE_LIMIT;
    if (sa.ax[0].k == 4 && sa.ax[1].k == 4 && sa.ax[2].k == 4) return INTERP_SPLINE4;
    return INTERP_SPLINE;
  }

  const DevGrid<T> &dgrid(const DiagT &d) const { return d.lg ? d.lg->dg : dg_; }
  long dN(const DiagT &d) const { return d.lg ? d.lg->N : N_; }
  long dT(const DiagT &d) const { return d.lg ? d.lg->ntot : ntot_; }
  static dim3 node_grid(const DevGrid<T> &g) { return dim3((g.P.n[0] + 31) / 32, (g.P.n[1] + 7) / 8, g.P.n[2]); }

  // new_sgrid_from_sgrid (src/sgrid_m.f90:446-761) for this library's tensor-product grids,
  // per axis: res > 0 puts res points between neighbouring nodes, x(ii) + dx * ir with
  // dx = (x(ii+1) - x(ii)) / (res+1) (the ghost image past the last node where the axis is
  // periodic, no points past it otherwise); res < 0 keeps every (|res|+1)-th node; singleton
  // axes stay.  Each new point inherits the flag of the node it starts from.  |res| >= n on a
  // non-singleton axis resets res to 0 (no new grid), as the reference does.  The new grid
  // goes through the same host set-up as the solver grid, then every lcs node is tracked to
  // the solver grid.
  bool make_lcs_grid(DiagT &d, int type, int &res, std::string &msg) {
    if (hg_.P.curv && res != 0) {
      msg = "diagnostic_init: resolution /= 0 on a non-rectilinear grid is not supported";
      return false;
    }
    for (int a = 0; a < 3; a++)
      if (n_[a] > 1 && std::abs(res) >= n_[a]) res = 0;
    if (res == 0) return true;
    std::vector<lcsdata_t> line[3];
    std::vector<int> src[3];  // solver index each new point starts from
    for (int a = 0; a < 3; a++) {
      const int n = n_[a];
      if (n == 1) {
        line[a].push_back(hg_.lt[a][1]);
        src[a].push_back(1);
        continue;
      }
      const int e1[3] = {a == 0 ? 1 : 0, a == 1 ? 1 : 0, a == 2 ? 1 : 0};
      for (int i = 1; i <= n; i++) {
        if (res > 0) {
          const lcsdata_t xi = hg_.coord(a, i * e1[0] + (1 - e1[0]), i * e1[1] + (1 - e1[1]), i * e1[2] + (1 - e1[2]));
          const lcsdata_t xn = hg_.coord(a, (i + 1) * e1[0] + (1 - e1[0]), (i + 1) * e1[1] + (1 - e1[1]), (i + 1) * e1[2] + (1 - e1[2]));
          const lcsdata_t dx = (xn - xi) / (lcsdata_t)(res + 1);
          for (int r = 0; r <= res; r++) {
            if (r > 0 && !hg_.P.per[a] && i == n) continue;
            line[a].push_back(xi + dx * (lcsdata_t)r);
            src[a].push_back(i);
          }
        } else if (i % (std::abs(res) + 1) == 0) {
          line[a].push_back(hg_.lt[a][i]);
          src[a].push_back(i);
        }
      }
    }
    const int nn[3] = {(int)line[0].size(), (int)line[1].size(), (int)line[2].size()};
    std::vector<int> F((size_t)nn[0] * nn[1] * nn[2]);
    for (int k = 0; k < nn[2]; k++)
      for (int j = 0; j < nn[1]; j++)
        for (int i = 0; i < nn[0]; i++)
          F[i + (size_t)nn[0] * (j + (size_t)nn[1] * k)] =
              (*out_flags_)[(src[0][i] - 1) + (size_t)n_[0] * ((src[1][j] - 1) + (size_t)n_[1] * (src[2][k] - 1))];
    return lcs_grid_from_lines(d, line, F, type, msg);
  }

  // An lcs grid from its coordinate lines and interior flags: host set-up, device tables, and
  // every node tracked to the solver grid (forward sets with the periodic wrap).
  bool lcs_grid_from_lines(DiagT &d, const std::vector<lcsdata_t> line[3], const std::vector<int> &F, int type, std::string &msg) {
    auto lg = std::make_shared<LcsGrid<T>>();
    const int nn[3] = {(int)line[0].size(), (int)line[1].size(), (int)line[2].size()};
    const long N = (long)nn[0] * nn[1] * nn[2];
    std::vector<lcsdata_t> X(N), Y(N), Z(N);
    for (int k = 0; k < nn[2]; k++)
      for (int j = 0; j < nn[1]; j++)
        for (int i = 0; i < nn[0]; i++) {
          const long q = i + (long)nn[0] * (j + (long)nn[1] * k);
          X[q] = line[0][i];
          Y[q] = line[1][j];
          Z[q] = line[2][k];
        }
    if (!lg->hg.build(nn, X.data(), Y.data(), Z.data(), F.data())) {
      msg = lg->hg.error;
      return false;
    }
    for (int a = 0; a < 3; a++) lg->out_lines[a] = std::make_shared<std::vector<double>>(line[a].begin(), line[a].end());
    lg->out_flags = std::make_shared<std::vector<int8_t>>(F.begin(), F.end());
    if (!make_dev_grid(lg->hg, lg->dg, msg)) return false;
    lg->N = N;
    lg->ntot = lg->hg.ntot();
    FieldPtrsW<T> pos{};
    for (int c = 0; c < 3; c++) {
      if (!(lg->pos[c] = arena_.alloc<T>(N, msg))) return false;
      if (!(lg->nos_reset[c] = arena_.alloc<int>(N, msg))) return false;
      if (!(lg->nos[c] = arena_.alloc<int>(N, msg))) return false;
      pos.f[c] = lg->pos[c];
    }
    k_track_lcs_nodes<T><<<node_grid(lg->dg), dim3(32, 8, 1), 0, stream_>>>(dg_, lg->dg, pos, lg->nos_reset[0], lg->nos_reset[1],
                                                                             lg->nos_reset[2], type == FTLE_FWD ? 1 : 0, &red_->err);
    CK(cudaGetLastError());
    counters_.kernel_launches++;
    d.lg = lg;
    return true;
  }

  // create_aux_grid (src/lcs_m.f90:225-435) for diagnostic diags_[pi]: per node, 0.2
  // (AUX_GRID_SCALING) times the mean distance to its in-bounds face neighbours; six copies of
  // the nodes shifted by -/+ that along x, y, z (projected back into the data plane on a 2-D
  // grid), each the nodes of an auxiliary grid with the lcs grid's flags and a particle set of
  // its own.  The device keeps coordinate lines, so each auxiliary grid must be a tensor
  // product to rounding (uniform spacing around every node, as on a cube); the per-node
  // separations of each pair are kept exactly for the gradient.
  bool create_aux(int pi, std::string &msg) {
    if (hg_.P.curv) {
      msg = "AUX_GRID: not supported on a non-rectilinear grid";
      return false;
    }
    const DiagT par = diags_[pi];  // copy: diags_ grows below
    const HostGrid<lcsdata_t> &bg = par.lg ? par.lg->hg : hg_;
    const int n[3] = {bg.P.n[0], bg.P.n[1], bg.P.n[2]};
    const long N = (long)n[0] * n[1] * n[2];
    static const int face[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    std::vector<lcsdata_t> delta(N), x3[6][3];
    std::vector<int> F(N);
    long q = 0;
    for (int k = 1; k <= n[2]; k++)
      for (int j = 1; j <= n[1]; j++)
        for (int i = 1; i <= n[0]; i++, q++) {
          lcsdata_t nbrsum = 0, distsum = 0;
          for (int nb = 0; nb < 6; nb++) {
            const int ii = i + face[nb][0], jj = j + face[nb][1], kk = k + face[nb][2];
            if (ii > 0 && jj > 0 && kk > 0 && ii <= n[0] && jj <= n[1] && kk <= n[2]) {
              nbrsum = nbrsum + lcsdata_t(1);
              const lcsdata_t dx = bg.coord(0, i, j, k) - bg.coord(0, ii, jj, kk), dy = bg.coord(1, i, j, k) - bg.coord(1, ii, jj, kk),
                              dz = bg.coord(2, i, j, k) - bg.coord(2, ii, jj, kk);
              distsum = distsum + std::sqrt(dx * dx + dy * dy + dz * dz);
            }
          }
          delta[q] = distsum / nbrsum * lcsdata_t(0.2);
          F[q] = bg.flag.empty() ? 0 : (int)bg.flag[bg.pidx(i, j, k)];
        }
    const int sa = bg.P.single_axis;
    for (int m = 0; m < 6; m++) {
      const int a = m % 3;
      for (int c = 0; c < 3; c++) x3[m][c].resize(N);
      q = 0;
      for (int k = 1; k <= n[2]; k++)
        for (int j = 1; j <= n[1]; j++)
          for (int i = 1; i <= n[0]; i++, q++) {
            for (int c = 0; c < 3; c++) x3[m][c][q] = bg.coord(c, i, j, k);
            x3[m][a][q] = m < 3 ? x3[m][a][q] - delta[q] : x3[m][a][q] + delta[q];
            // project_lp2plane on an axis-aligned plane: x - ((x - x_node) . n) n
            if (sa >= 0) x3[m][sa][q] = x3[m][sa][q] - (x3[m][sa][q] - bg.coord(sa, i, j, k));
          }
    }
    // each auxiliary grid's coordinate lines (first row), checked against every node
    std::vector<int> idx;
    for (int m = 0; m < 6; m++) {
      std::vector<lcsdata_t> line[3];
      for (int i = 0; i < n[0]; i++) line[0].push_back(x3[m][0][i]);
      for (int j = 0; j < n[1]; j++) line[1].push_back(x3[m][1][(size_t)n[0] * j]);
      for (int k = 0; k < n[2]; k++) line[2].push_back(x3[m][2][(size_t)n[0] * n[1] * k]);
      lcsdata_t span = 0, dev = 0;
      q = 0;
      for (int k = 0; k < n[2]; k++)
        for (int j = 0; j < n[1]; j++)
          for (int i = 0; i < n[0]; i++, q++) {
            const int id[3] = {i, j, k};
            for (int c = 0; c < 3; c++) {
              dev = std::max(dev, (lcsdata_t)std::fabs((double)(x3[m][c][q] - line[c][id[c]])));
              span = std::max(span, (lcsdata_t)std::fabs((double)x3[m][c][q]));
            }
          }
      if (dev > lcsdata_t(64) * std::numeric_limits<lcsdata_t>::epsilon() * std::max(span, lcsdata_t(1))) {
        msg = "AUX_GRID: an auxiliary grid is not a tensor product (the grid spacing differs around some node); "
              "this library supports AUX_GRID on uniformly spaced grids only";
        return false;
      }
      DiagT A;
      A.handle = 0;
      A.type = par.type;
      A.T_ = par.T_;
      A.h = par.h;
      A.dt_factor = par.dt_factor;
      A.nslot = par.nslot;
      A.aux_parent = pi + 1;
      if (!lcs_grid_from_lines(A, line, F, par.type, msg)) return false;
      if (!alloc_diag(A, msg)) return false;
      diags_.push_back(A);
      idx.push_back((int)diags_.size() - 1);
    }
    DiagT &P = diags_[pi];
    P.aux = idx;
    for (int a = 0; a < 3; a++) {
      std::vector<lcsdata_t> den(N);
      for (long r = 0; r < N; r++) den[r] = x3[a + 3][a][r] - x3[a][a][r];
      if (!(P.auxden[a] = upload(den, msg))) return false;
    }
    if (cudaStreamSynchronize(stream_) != cudaSuccess) {
      msg = "CUDA error in sync";
      return false;
    }
    return true;
  }

  bool launch_ftle_aux(DiagT &d, std::string &msg) {
    const DevGrid<T> &g = dgrid(d);
    AuxMaps<T> M{};
    for (int a = 0; a < 3; a++) {
      for (int c = 0; c < 3; c++) {
        M.lo[a][c] = diags_[d.aux[a]].composed[c];
        M.hi[a][c] = diags_[d.aux[a + 3]].composed[c];
      }
      M.den[a] = d.auxden[a];
    }
    counters_.kernel_launches++;
    k_ftle_aux<T, lcsdata_t><<<node_grid(g), dim3(32, 8, 1), 0, stream_>>>(g, M, d.ftle, d.T_, opt_->incompressible);
    CK(cudaGetLastError());
    return true;
  }

  // backward sets: the working solver nodes back to the tracked ones (reset_lp + track_lp2node)
  bool reset_refined_nodes(DiagT &d, std::string &msg) {
    for (int c = 0; c < 3; c++)
      CK(cudaMemcpyAsync(d.lg->nos[c], d.lg->nos_reset[c], d.lg->N * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
    return true;
  }

  template <int INTERP, bool FS, bool FL>
  void sl_refined_integ(DiagT &d, const SplineAxes<T> &sas, const SplineAxes<T> &sal, const VelFields<TV> &V, FieldPtrs<T> fo,
                        FieldPtrsW<T> fn, StageTimes S, T dt) {
    LcsGrid<T> &L = *d.lg;
    FieldPtrs<T> pos{};
    for (int c = 0; c < 3; c++) pos.f[c] = L.pos[c];
    const dim3 grd = node_grid(L.dg), blk(32, 8, 1);
    int *err = &red_->err;
    counters_.kernel_launches++;
#define SLR(IG)                                                                                                   \
  k_sl_refined<T, TV, IG, INTERP, FS, FL><<<grd, blk, 0, stream_>>>(L.dg, dg_, sas, sal, pos, L.nos[0], L.nos[1], L.nos[2], V, fo, fn, \
                                                                     S, dt, err)
    switch (opt_->integrator) {
      case 0: SLR(EULER_); break;
      case 1: SLR(TRAPEZOIDAL_); break;
      case 2: SLR(RK2_); break;
      case 3: SLR(RK3_); break;
      default: SLR(RK4_); break;
    }
#undef SLR
  }

  template <int INTERP>
  void sl_refined_flags(DiagT &d, const SplineAxes<T> &sas, const SplineAxes<T> &sal, const VelFields<TV> &V, FieldPtrs<T> fo,
                        FieldPtrsW<T> fn, StageTimes S, T dt) {
    const bool FS = dg_.P.has_flags != 0, FL = d.lg->dg.P.has_flags != 0;
    if (FS && FL) sl_refined_integ<INTERP, true, true>(d, sas, sal, V, fo, fn, S, dt);
    else if (FS) sl_refined_integ<INTERP, true, false>(d, sas, sal, V, fo, fn, S, dt);
    else if (FL) sl_refined_integ<INTERP, false, true>(d, sas, sal, V, fo, fn, S, dt);
    else sl_refined_integ<INTERP, false, false>(d, sas, sal, V, fo, fn, S, dt);
  }

  // sas: the solver grid's spline axes (velocity), sal: the lcs grid's (flow map); the kernel
  // takes the all-cubic specialisation only when both grids allow it
  bool launch_sl_refined(DiagT &d, const SplineAxes<T> &sas, const SplineAxes<T> &sal, const VelFields<TV> &V, FieldPtrs<T> fo,
                         FieldPtrsW<T> fn, StageTimes S, T dt, std::string &msg) {
    const int interp = interpolator();
    if (interp == NEAREST_NBR) sl_refined_flags<INTERP_NEAREST>(d, sas, sal, V, fo, fn, S, dt);
    else if (interp == LINEAR) sl_refined_flags<INTERP_LINEAR>(d, sas, sal, V, fo, fn, S, dt);
    else if (interp == TSE) sl_refined_flags<INTERP_TSE>(d, sas, sal, V, fo, fn, S, dt);
    else if (interp == TSE_LIMIT) sl_refined_flags<INTERP_TSE_LIMIT>(d, sas, sal, V, fo, fn, S, dt);
    else if (interp_variant(interp, sas) == INTERP_SPLINE4 && interp_variant(interp, sal) == INTERP_SPLINE4)
      sl_refined_flags<INTERP_SPLINE4>(d, sas, sal, V, fo, fn, S, dt);
    else sl_refined_flags<INTERP_SPLINE>(d, sas, sal, V, fo, fn, S, dt);
    CK(cudaGetLastError());
    return true;
  }

  // Device tables of a host grid set-up (coordinate lines, spans, flags, normals, constants)
  bool make_dev_grid(const HostGrid<lcsdata_t> &hg, DevGrid<T> &dg, std::string &msg) {
    GridParams<T> P{};
    const GridParams<lcsdata_t> &H = hg.P;
    for (int a = 0; a < 3; a++) {
      P.n[a] = H.n[a];
      P.per[a] = H.per[a];
      for (int s = 0; s < 2; s++)
        for (int e = 0; e < 2; e++) P.gx[a][s][e] = (T)H.gx[a][s][e];
    }
    P.sx = H.sx;
    P.sxy = H.sxy;
    P.single_axis = H.single_axis;
    P.zquirk = H.zquirk;
    for (int q = 0; q < 6; q++) P.bb[q] = (T)H.bb[q];
    for (int d = 0; d < 27; d++)
      for (int c = 0; c < 3; c++) P.ps[d][c] = (T)H.ps[d][c];
    P.has_flags = H.has_flags;
    P.maxtrack = H.maxtrack;
    P.curv = H.curv;
    for (int a = 0; a < 3; a++) {
      P.guess0[a] = H.guess0[a];
      for (int c = 0; c < 3; c++) P.guessd[a][c] = (T)H.guessd[a][c];
    }
    dg.P = P;
    for (int a = 0; a < 3; a++) {
      if (!(dg.lt[a] = upload(hg.lt[a], msg))) return false;
      if (!(dg.li[a] = upload(hg.li[a], msg))) return false;
      if (!(dg.ri[a] = upload(reciprocal_spans(hg.li[a]), msg))) return false;
      if (!(dg.invd[a] = upload(hg.invd[a], msg))) return false;
    }
    dg.lsw = nullptr;
    for (int a = 0; a < 3; a++) dg.X[a] = dg.pnrm[a] = dg.invdp[a] = nullptr;
    if (H.curv) {
      for (int a = 0; a < 3; a++) {
        if (!(dg.X[a] = upload(hg.X[a], msg))) return false;
        if (!(dg.invdp[a] = upload(hg.invdp[a], msg))) return false;
        if (!hg.pnorm[a].empty() && !(dg.pnrm[a] = upload(hg.pnorm[a], msg))) return false;
      }
      if (!(dg.lsw = upload(hg.lsw, msg))) return false;
    }
    dg.flag = nullptr;
    for (int a = 0; a < 3; a++) dg.nrm[a] = nullptr;
    if (H.has_flags) {
      int8_t *f = arena_.alloc<int8_t>(hg.flag.size(), msg);
      if (!f) return false;
      CK(cudaMemcpy(f, hg.flag.data(), hg.flag.size(), cudaMemcpyHostToDevice));
      dg.flag = f;
      if (!hg.bcnorm.empty()) {
        for (int a = 0; a < 3; a++) {
          std::vector<lcsdata_t> comp(hg.bcnorm.begin() + (size_t)a * hg.ntot(), hg.bcnorm.begin() + (size_t)(a + 1) * hg.ntot());
          if (!(dg.nrm[a] = upload(comp, msg))) return false;
        }
      } else {
        // flags without normals (e.g. only INFLOW/OUTFLOW or 2-D): a zero field keeps the
        // kernels free of null checks
        std::vector<lcsdata_t> zero(hg.ntot(), lcsdata_t(0));
        T *z0 = upload(zero, msg);
        if (!z0) return false;
        for (int a = 0; a < 3; a++) dg.nrm[a] = z0;
      }
    }
    return true;
  }

  dim3 node_grid() const { return dim3((n_[0] + 31) / 32, (n_[1] + 7) / 8, n_[2]); }

  // Subcycle kernels that stage their taps in shared memory (k_sl_tile, k_sl_tile_lin,
  // k_fwd_tile) are bitwise equal to the gathering kernels they replace, so which of the two runs
  // is a question of speed only, and the engine measures it: for the backward kernel (family 0)
  // and the forward kernel (family 1) it alternates the two variants -- launch by launch, or
  // sort interval by sort interval for the forward kernel, whose staged variant needs its own
  // sort tiles -- times each launch with the CUDA events that bracket it, and once each variant
  // has kTuneSamples launches keeps the one with the shorter launch for the rest of the engine's
  // life (per instance: the batched form tunes every instance for its own grid and options).
  // Measured on B200, ABC 256^3 FP64 per launch: staged cubic backward 3.14 against 4.44 ms,
  // staged forward 5.93 against 4.88 ms (first launches), staged LINEAR backward (the z-marching
  // kernel) 0.55 against 0.84 ms.
  // CFD2LCS_B200_SL_TILE at cfd2lcs_init: 0 = gathering kernels only, 1 = tuned (default),
  // 2 = staged kernels wherever they apply.  cfd2lcs_get_tuning_c reports the choices.
  // Each variant's first launch is dropped and the rest compared by their minimum: a launch whose
  // events also bracket host set-up (cudaFuncSetAttribute, the first encoding of a buffer's
  // tensor map) while the GPU idles can only read long, and such launches come first.
  static constexpr int kTuneSamples = 6;
  int tile_mode_ = 1;
  struct Tuner {
    int choice = -1;  // -1: sampling, 0: gathering, 1: staged
    double ms[2] = {1e300, 1e300};  // smallest launch time per variant
    int n[2] = {0, 0};              // launches seen per variant
  } tune_[2];
  long tune_idx_[2] = {0, 0};

  // the variant of the next launch (or sort interval) of family fam, for which staging applies
  int tile_variant(int fam) {
    if (tile_mode_ != 1) return tile_mode_ == 2 ? 1 : 0;
    if (tune_[fam].choice >= 0) return tune_[fam].choice;
    return (int)(tune_idx_[fam]++ & 1);
  }

  void tune_record(int tag, double ms) {
    Tuner &t = tune_[tag / 2];
    const int v = tag % 2;
    if (t.choice >= 0) return;
    if (t.n[v]++ > 0) t.ms[v] = std::min(t.ms[v], ms);
    if (t.n[0] > kTuneSamples && t.n[1] > kTuneSamples) t.choice = t.ms[1] < t.ms[0] ? 1 : 0;
  }

  void tuning(int choice[2], double ms[4]) const override {
    for (int f = 0; f < 2; f++) {
      choice[f] = tune_[f].choice;
      for (int v = 0; v < 2; v++) ms[2 * f + v] = tune_[f].n[v] > 1 ? tune_[f].ms[v] : 0.0;
    }
  }

  int sl_variant_ = -1;  // variant of the last backward launch while sampling (-1: none)

  // Tensor maps of the staged fields (one per padded component buffer and box shape), so that a
  // block copies each component's box with one cp.async.bulk.tensor instead of one bulk copy per
  // row; CFD2LCS_B200_TMA_TENSOR=0 at cfd2lcs_init keeps the row copies.  A map needs rows of a
  // multiple of 16 bytes (padded x extent * element size); other grids copy rows.
  bool tma_tensor_ = true;
  std::map<std::array<uintptr_t, 5>, CUtensorMap> tmaps_;

  template <typename TC>
  bool tensor_map(const TC *ptr, int bx, int by, int bz, CUtensorMap &out) {
    if (!tma_tensor_ || !ptr) return false;
    const long sx = dg_.P.sx, sxy = dg_.P.sxy, es = (long)sizeof(TC);
    if ((sx * es) % 16 || reinterpret_cast<uintptr_t>(ptr) % 16) return false;
    const std::array<uintptr_t, 5> key = {reinterpret_cast<uintptr_t>(ptr), (uintptr_t)es, (uintptr_t)bx, (uintptr_t)by, (uintptr_t)bz};
    auto it = tmaps_.find(key);
    if (it != tmaps_.end()) {
      out = it->second;
      return true;
    }
    const EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return false;
    const cuuint64_t dim[3] = {(cuuint64_t)sx, (cuuint64_t)(sxy / sx), (cuuint64_t)(n_[2] + 2)};
    const cuuint64_t stride[2] = {(cuuint64_t)(sx * es), (cuuint64_t)(sxy * es)};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz}, estr[3] = {1, 1, 1};
    CUtensorMap m;
    if (fn(&m, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<TC *>(ptr), dim, stride, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    tmaps_[key] = m;
    out = m;
    return true;
  }

  // the maps of fields f0..: three component pointers each, boxes of geometry G
  template <typename G, typename TC>
  bool tensor_maps3(const TC *const f[3], CUtensorMap *out) {
    for (int c = 0; c < 3; c++)
      if (!tensor_map<TC>(f[c], G::template pitch<TC>(), G::SY, G::SZ, out[c])) return false;
    return true;
  }
  int dev_ = 0;  // CUDA device current at cfd2lcs_init

  template <int IG, bool F>
  void launch_sl_tile(const SplineAxes<T> &sa, const VelFields<TV> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn, StageTimes S, T dt) {
    const size_t smem = slt_field_bytes<T>() + 128;
    cudaFuncSetAttribute(k_sl_tile<T, TV, IG, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 blk(32, SLT_Y, 2), grd((n_[0] + SLT_X - 1) / SLT_X, (n_[1] + SLT_Y - 1) / SLT_Y, (n_[2] + SLT_Z - 1) / SLT_Z);
    constexpr int noff = IG == RK2_ ? 1 : (IG == RK3_ ? 2 : (IG == RK4_ ? 3 : 0));
    TileMaps tm{};
    bool ok = true;
    for (int f = 0; f < noff && ok; f++) ok = tensor_maps3<CubicGeom, TV>(V.cs[f + 1], tm.m + 3 * f);
    ok = ok && tensor_maps3<CubicGeom, T>(fo.f, tm.m + 3 * noff);
    tm.on = ok ? 1 : 0;
    k_sl_tile<T, TV, IG, F><<<grd, blk, smem, stream_>>>(dg_, sa, V, fo, fn, S, dt, &red_->err, tm);
  }

  // the bulk copies need 16-byte aligned sources (cudaMalloc gives 256)
  bool sl_tile_usable(const VelFields<TV> &V, FieldPtrs<T> fo) const {
    if (!tile_mode_) return false;
    const int noff = opt_->integrator == 2 ? 1 : (opt_->integrator == 3 ? 2 : (opt_->integrator == 4 ? 3 : 0));
    for (int c = 0; c < 3; c++) {
      if (reinterpret_cast<uintptr_t>(fo.f[c]) % 16) return false;
      for (int s = 1; s <= noff; s++)
        if (!V.cs[s][c] || reinterpret_cast<uintptr_t>(V.cs[s][c]) % 16) return false;
    }
    return true;
  }

  // The staged LINEAR backward kernel: k_sl_march_lin (planes marching along z) where every
  // field has a tensor map and the velocity is stored in the flow map's type, else the boxes of
  // k_sl_tile_lin.  CFD2LCS_B200_SL_MARCH=0 at cfd2lcs_init keeps the boxes;
  // CFD2LCS_B200_SL_MARCH_KC sets the planes per column run (default: runs of 8..64 planes
  // giving about eight waves of two blocks per SM).
  bool sl_march_ = true;
  int sl_march_kc_ = 0;
  int num_sms_ = 148;

  template <int IG, bool F>
  bool launch_sl_march_lin(const VelFields<TV> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn, StageTimes S, T dt) {
    if constexpr (!std::is_same<T, TV>::value) {
      return false;
    } else {
      // a box row (SLM_SX elements) must be a multiple of 16 bytes: FP64 only
      if (!sl_march_ || (SLM_SX * sizeof(T)) % 16) return false;
      TileMaps tm{};
      for (int c = 0; c < 3; c++)
        if (!tensor_map<T>(V.un[c], SLM_SX, SLM_SY, 1, tm.m[c]) || !tensor_map<T>(V.unp1[c], SLM_SX, SLM_SY, 1, tm.m[3 + c]) ||
            !tensor_map<T>(fo.f[c], SLM_SX, SLM_SY, 1, tm.m[6 + c]))
          return false;
      tm.on = 1;
      const long cols = (long)((n_[0] + SLM_X - 1) / SLM_X) * ((n_[1] + SLM_Y - 1) / SLM_Y);
      int kc = sl_march_kc_;
      if (kc <= 0) kc = (int)std::max(8L, std::min(64L, (long)n_[2] * cols / (8L * 2 * num_sms_)));
      kc = std::min(kc, n_[2]);
      const size_t smem = slm_bytes<T>() + 128;
      cudaFuncSetAttribute(k_sl_march_lin<T, IG, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      const dim3 blk(SLM_X, SLM_Y, 1), grd((n_[0] + SLM_X - 1) / SLM_X, (n_[1] + SLM_Y - 1) / SLM_Y, (n_[2] + kc - 1) / kc);
      k_sl_march_lin<T, IG, F><<<grd, blk, smem, stream_>>>(dg_, fn, S, dt, kc, &red_->err, tm);
      counters_.sl_march_launches++;
      return true;
    }
  }

  template <int IG, bool F>
  void launch_sl_tile_lin(const VelFields<TV> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn, StageTimes S, T dt) {
    if (launch_sl_march_lin<IG, F>(V, fo, fn, S, dt)) return;
    const size_t smem = sll_bytes<T, TV>() + 128;
    cudaFuncSetAttribute(k_sl_tile_lin<T, TV, IG, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const dim3 blk(32, LinGeom::TY, 2),
        grd((n_[0] + LinGeom::TX - 1) / LinGeom::TX, (n_[1] + LinGeom::TY - 1) / LinGeom::TY, (n_[2] + LinGeom::TZ - 1) / LinGeom::TZ);
    TileMaps tm{};
    tm.on = tensor_maps3<LinGeom, TV>(V.un, tm.m) && tensor_maps3<LinGeom, TV>(V.unp1, tm.m + 3) && tensor_maps3<LinGeom, T>(fo.f, tm.m + 6)
                ? 1
                : 0;
    k_sl_tile_lin<T, TV, IG, F><<<grd, blk, smem, stream_>>>(dg_, V, fo, fn, S, dt, &red_->err, tm);
  }

  // LINEAR: 3-D grids whose backward set samples both levels per corner (no stage blends)
  bool sl_tile_lin_usable(const VelFields<TV> &V, FieldPtrs<T> fo) const {
    if (!tile_mode_ || n_[2] < 4 || dg_.P.single_axis >= 0 || !dg_.ri[0] || !dg_.ri[1] || !dg_.ri[2]) return false;
    for (int c = 0; c < 3; c++) {
      if (V.cs[1][c] || reinterpret_cast<uintptr_t>(fo.f[c]) % 16 || reinterpret_cast<uintptr_t>(V.un[c]) % 16 ||
          reinterpret_cast<uintptr_t>(V.unp1[c]) % 16)
        return false;
    }
    return true;
  }

  template <int INTERP, bool F>
  void sl_integ(const SplineAxes<T> &sa, const VelFields<TV> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn, StageTimes S, T dt) {
    sl_variant_ = -1;
    if constexpr (INTERP == INTERP_LINEAR) {
      if (sl_tile_lin_usable(V, fo) && (sl_variant_ = tile_variant(0)) == 1) {
        counters_.kernel_launches++;
        counters_.sl_staged_launches++;
        switch (opt_->integrator) {
          case 0: launch_sl_tile_lin<EULER_, F>(V, fo, fn, S, dt); break;
          case 1: launch_sl_tile_lin<TRAPEZOIDAL_, F>(V, fo, fn, S, dt); break;
          case 2: launch_sl_tile_lin<RK2_, F>(V, fo, fn, S, dt); break;
          case 3: launch_sl_tile_lin<RK3_, F>(V, fo, fn, S, dt); break;
          default: launch_sl_tile_lin<RK4_, F>(V, fo, fn, S, dt); break;
        }
        return;
      }
    }
    if constexpr (INTERP == INTERP_SPLINE4) {
      if (sl_tile_usable(V, fo) && (sl_variant_ = tile_variant(0)) == 1) {
        counters_.kernel_launches++;
        counters_.sl_staged_launches++;
        switch (opt_->integrator) {
          case 0: launch_sl_tile<EULER_, F>(sa, V, fo, fn, S, dt); break;
          case 1: launch_sl_tile<TRAPEZOIDAL_, F>(sa, V, fo, fn, S, dt); break;
          case 2: launch_sl_tile<RK2_, F>(sa, V, fo, fn, S, dt); break;
          case 3: launch_sl_tile<RK3_, F>(sa, V, fo, fn, S, dt); break;
          default: launch_sl_tile<RK4_, F>(sa, V, fo, fn, S, dt); break;
        }
        return;
      }
    }
    // blocks of 32 x 8/bz x bz nodes: spanning z layers lets a block's warps share the corners
    // of the layers between them in L1.  Measured on B200 (bz = 1 / 2 / 4): FP64 velocity, ABC
    // 256^3 CUBIC 4.30 / 4.12 / 4.10 ms and turbulence 512^3 LINEAR 7.84 / 7.64 / 7.50 ms per
    // launch; FP32 velocity, ABC 256^3 2.81 / 2.79 / 2.96 ms.  Flat blocks on 2-D grids.
    const int bz = n_[2] < 8 ? 1 : (std::is_same<TV, float>::value ? 2 : 4), by = 8 / bz;
    const dim3 blk(32, by, bz), grd((n_[0] + 31) / 32, (n_[1] + by - 1) / by, (n_[2] + bz - 1) / bz);
    int *err = &red_->err;
    counters_.kernel_launches++;
    switch (opt_->integrator) {
      case 0: k_sl_subcycle<T, TV, EULER_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case 1: k_sl_subcycle<T, TV, TRAPEZOIDAL_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case 2: k_sl_subcycle<T, TV, RK2_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      case 3: k_sl_subcycle<T, TV, RK3_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
      default: k_sl_subcycle<T, TV, RK4_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, fo, fn, S, dt, err); break;
    }
  }

  bool launch_sl(int iv, const SplineAxes<T> &sa, const VelFields<TV> &V, FieldPtrs<T> fo, FieldPtrsW<T> fn, StageTimes S, T dt,
                 std::string &msg) {
    const bool F = dg_.P.has_flags != 0;
    if (iv == INTERP_NEAREST) F ? sl_integ<INTERP_NEAREST, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_NEAREST, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_LINEAR) F ? sl_integ<INTERP_LINEAR, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_LINEAR, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_TSE) F ? sl_integ<INTERP_TSE, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_TSE, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_TSE_LIMIT) F ? sl_integ<INTERP_TSE_LIMIT, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_TSE_LIMIT, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_CTSE) F ? sl_integ<INTERP_CTSE, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_CTSE, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_CTSE_LIMIT)
      F ? sl_integ<INTERP_CTSE_LIMIT, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_CTSE_LIMIT, false>(sa, V, fo, fn, S, dt);
    else if (iv == INTERP_SPLINE4) F ? sl_integ<INTERP_SPLINE4, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_SPLINE4, false>(sa, V, fo, fn, S, dt);
    else F ? sl_integ<INTERP_SPLINE, true>(sa, V, fo, fn, S, dt) : sl_integ<INTERP_SPLINE, false>(sa, V, fo, fn, S, dt);
    CK(cudaGetLastError());
    return true;
  }

  template <int INTERP, bool F>
  void fwd_integ(const SplineAxes<T> &sa, const VelFields<TV> &V, Particles<T> P, StageTimes S, T dt, int np) {
    const int blk = 256, grd = (int)((np + blk - 1) / blk);
    int *err = &red_->err;
    counters_.kernel_launches++;
    switch (opt_->integrator) {
      case 0: k_fwd_subcycle<T, TV, EULER_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, P, S, dt, np, err); break;
      case 1: k_fwd_subcycle<T, TV, TRAPEZOIDAL_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, P, S, dt, np, err); break;
      case 2: k_fwd_subcycle<T, TV, RK2_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, P, S, dt, np, err); break;
      case 3: k_fwd_subcycle<T, TV, RK3_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, P, S, dt, np, err); break;
      default: k_fwd_subcycle<T, TV, RK4_, INTERP, F><<<grd, blk, 0, stream_>>>(dg_, sa, V, P, S, dt, np, err); break;
    }
  }

  bool launch_fwd(int iv, const SplineAxes<T> &sa, const VelFields<TV> &V, Particles<T> P, StageTimes S, T dt, std::string &msg,
                  long np = -1) {
    const bool F = dg_.P.has_flags != 0;
    const int n = (int)(np < 0 ? N_ : np);
    if (n == 0) return true;
    if (iv == INTERP_NEAREST) F ? fwd_integ<INTERP_NEAREST, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_NEAREST, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_LINEAR) F ? fwd_integ<INTERP_LINEAR, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_LINEAR, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_TSE) F ? fwd_integ<INTERP_TSE, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_TSE, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_TSE_LIMIT) F ? fwd_integ<INTERP_TSE_LIMIT, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_TSE_LIMIT, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_CTSE) F ? fwd_integ<INTERP_CTSE, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_CTSE, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_CTSE_LIMIT)
      F ? fwd_integ<INTERP_CTSE_LIMIT, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_CTSE_LIMIT, false>(sa, V, P, S, dt, n);
    else if (iv == INTERP_SPLINE4) F ? fwd_integ<INTERP_SPLINE4, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_SPLINE4, false>(sa, V, P, S, dt, n);
    else F ? fwd_integ<INTERP_SPLINE, true>(sa, V, P, S, dt, n) : fwd_integ<INTERP_SPLINE, false>(sa, V, P, S, dt, n);
    CK(cudaGetLastError());
    return true;
  }

  // The cubic forward subcycle with its taps staged in shared memory (k_fwd_tile): sorted
  // particle sets on 3-D grids, unless CFD2LCS_B200_SL_TILE=0 at cfd2lcs_init.
  bool fwd_tile_usable(int iv, const VelFields<TV> &V) const {
    if (!tile_mode_ || iv != INTERP_SPLINE4) return false;
    const int ns = opt_->integrator == 2 ? 2 : (opt_->integrator == 3 ? 3 : (opt_->integrator == 4 ? 4 : 1));
    for (int s = 0; s < ns; s++)
      for (int c = 0; c < 3; c++)
        if (!V.cs[s][c] || reinterpret_cast<uintptr_t>(V.cs[s][c]) % 16) return false;
    return true;
  }

  template <int IG, bool F>
  void fwd_tile_integ(const SplineAxes<T> &sa, const VelFields<TV> &V, DiagT &d, StageTimes S, T dt) {
    const size_t smem = fwt_bytes<TV>() + 128;
    cudaFuncSetAttribute(k_fwd_tile<T, TV, IG, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long ntiles = (long)d.sort_geom.ntx * d.sort_geom.nty * d.sort_geom.ntz;
    constexpr int ns = IG == RK2_ ? 2 : (IG == RK3_ ? 3 : (IG == RK4_ ? 4 : 1));
    TileMaps tm{};
    bool ok = true;
    for (int st = 0; st < ns && ok; st++) ok = tensor_maps3<FwdGeom, TV>(V.cs[st], tm.m + 3 * st);
    tm.on = ok ? 1 : 0;
    k_fwd_tile<T, TV, IG, F><<<(unsigned)ntiles, FWT_THREADS, smem, stream_>>>(dg_, sa, V, d.P, S, dt, d.poffs, d.ptsum, d.sort_geom,
                                                                              (int)dN(d), &red_->err, tm);
  }

  bool launch_fwd_tile(DiagT &d, const SplineAxes<T> &sa, const VelFields<TV> &V, StageTimes S, T dt, std::string &msg) {
    const bool F = dg_.P.has_flags != 0;
    counters_.kernel_launches++;
    counters_.fwd_staged_launches++;
    switch (opt_->integrator) {
      case 0: F ? fwd_tile_integ<EULER_, true>(sa, V, d, S, dt) : fwd_tile_integ<EULER_, false>(sa, V, d, S, dt); break;
      case 1: F ? fwd_tile_integ<TRAPEZOIDAL_, true>(sa, V, d, S, dt) : fwd_tile_integ<TRAPEZOIDAL_, false>(sa, V, d, S, dt); break;
      case 2: F ? fwd_tile_integ<RK2_, true>(sa, V, d, S, dt) : fwd_tile_integ<RK2_, false>(sa, V, d, S, dt); break;
      case 3: F ? fwd_tile_integ<RK3_, true>(sa, V, d, S, dt) : fwd_tile_integ<RK3_, false>(sa, V, d, S, dt); break;
      default: F ? fwd_tile_integ<RK4_, true>(sa, V, d, S, dt) : fwd_tile_integ<RK4_, false>(sa, V, d, S, dt); break;
    }
    CK(cudaGetLastError());
    return true;
  }

  bool launch_snapshot(DiagT &d, int s, std::string &msg) {
    const DevGrid<T> &g = dgrid(d);
    const dim3 blk(32, 8, 1), grd = node_grid(g);
    FieldPtrs<T> src{};
    FieldPtrsW<T> dst{};
    for (int c = 0; c < 3; c++) {
      dst.f[c] = d.slot[3 * s + c];
      src.f[c] = d.type == FTLE_BKWD ? d.fm[d.cur][c] : nullptr;
    }
    int *err = &red_->err;
    const bool F = g.P.has_flags != 0;
    counters_.kernel_launches++;
    if (d.type == FTLE_BKWD) {
      if (F) k_snapshot<T, true, false><<<grd, blk, 0, stream_>>>(g, src, d.P, dst, err);
      else k_snapshot<T, false, false><<<grd, blk, 0, stream_>>>(g, src, d.P, dst, err);
    } else {
      if (F) k_snapshot<T, true, true><<<grd, blk, 0, stream_>>>(g, src, d.P, dst, err);
      else k_snapshot<T, false, true><<<grd, blk, 0, stream_>>>(g, src, d.P, dst, err);
    }
    CK(cudaGetLastError());
    return true;
  }

  template <int I, bool FL>
  void compose_steps(const SplineAxes<T> &sa, DiagT &d, int m, FieldPtrsW<T> out) {
    const int np = (int)N_, grd = (np + 255) / 256;
    int *err = &red_->err;
    const SortTiles st = sort_tiles(n_, 32, SORT_TY, SORT_TZ);
    std::string dummy;
    k_reset_particles<T><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, cp_[0]);
    counters_.kernel_launches++;
    int cur = 0;
    for (int s = 0; s < m; s++) {
      if (s > 0 && s % compose_sort_every_ == 0) {
        sort_slots(cp_[cur], cp_[cur ^ 1], cp_key_, cp_cnt_, cp_offs_, cp_tsum_, np, st, dummy);
        cur ^= 1;
      }
      FieldPtrs<T> f{};
      for (int c = 0; c < 3; c++) f.f[c] = d.slot_list_host[3 * s + c];
      if (compose_minb_ == 4) k_compose_step<T, I, FL, 4><<<grd, 256, 0, stream_>>>(dg_, sa, f, cp_[cur], np, err);
      else k_compose_step<T, I, FL, 2><<<grd, 256, 0, stream_>>>(dg_, sa, f, cp_[cur], np, err);
      counters_.kernel_launches++;
    }
    k_compose_finish<T, FL><<<grd, 256, 0, stream_>>>(dg_, cp_[cur], out, np);
    counters_.kernel_launches++;
  }

  bool launch_compose(int iv, const SplineAxes<T> &sa, DiagT &d, int m, std::string &msg) {
    if (!d.lg && cp_[0].x[0] && N_ >= compose_sort_min_) {
      FieldPtrsW<T> out{};
      for (int c = 0; c < 3; c++) out.f[c] = d.composed[c];
      counters_.slots_composed += m;
      const bool F = dg_.P.has_flags != 0;
#define COMPOSE_STEPS(I) (F ? compose_steps<I, true>(sa, d, m, out) : compose_steps<I, false>(sa, d, m, out))
      if (iv == INTERP_NEAREST) COMPOSE_STEPS(INTERP_NEAREST);
      else if (iv == INTERP_LINEAR) COMPOSE_STEPS(INTERP_LINEAR);
      else if (iv == INTERP_TSE) COMPOSE_STEPS(INTERP_TSE);
      else if (iv == INTERP_TSE_LIMIT) COMPOSE_STEPS(INTERP_TSE_LIMIT);
      else if (iv == INTERP_CTSE) COMPOSE_STEPS(INTERP_CTSE);
      else if (iv == INTERP_CTSE_LIMIT) COMPOSE_STEPS(INTERP_CTSE_LIMIT);
      else if (iv == INTERP_SPLINE4) COMPOSE_STEPS(INTERP_SPLINE4);
      else COMPOSE_STEPS(INTERP_SPLINE);
#undef COMPOSE_STEPS
      CK(cudaGetLastError());
      return true;
    }
    const DevGrid<T> &g = dgrid(d);
    const dim3 blk(32, 8, 1), grd = node_grid(g);
    FieldPtrsW<T> out{};
    for (int c = 0; c < 3; c++) out.f[c] = d.composed[c];
    int *err = &red_->err;
    const bool F = g.P.has_flags != 0;
    const T *const *sl = d.slot_list_dev;
    counters_.kernel_launches++;
    counters_.slots_composed += m;
#define COMPOSE(I, FL) k_compose<T, I, FL><<<grd, blk, 0, stream_>>>(g, sa, sl, m, out, err)
    if (iv == INTERP_NEAREST) { if (F) COMPOSE(INTERP_NEAREST, true); else COMPOSE(INTERP_NEAREST, false); }
    else if (iv == INTERP_LINEAR) { if (F) COMPOSE(INTERP_LINEAR, true); else COMPOSE(INTERP_LINEAR, false); }
    else if (iv == INTERP_TSE) { if (F) COMPOSE(INTERP_TSE, true); else COMPOSE(INTERP_TSE, false); }
    else if (iv == INTERP_TSE_LIMIT) { if (F) COMPOSE(INTERP_TSE_LIMIT, true); else COMPOSE(INTERP_TSE_LIMIT, false); }
    else if (iv == INTERP_CTSE) { if (F) COMPOSE(INTERP_CTSE, true); else COMPOSE(INTERP_CTSE, false); }
    else if (iv == INTERP_CTSE_LIMIT) { if (F) COMPOSE(INTERP_CTSE_LIMIT, true); else COMPOSE(INTERP_CTSE_LIMIT, false); }
    else if (iv == INTERP_SPLINE4) { if (F) COMPOSE(INTERP_SPLINE4, true); else COMPOSE(INTERP_SPLINE4, false); }
    else { if (F) COMPOSE(INTERP_SPLINE, true); else COMPOSE(INTERP_SPLINE, false); }
#undef COMPOSE
    CK(cudaGetLastError());
    return true;
  }

  // k_ftle for the grid's form: flags or not, central differences or least squares (curvilinear)
  void launch_ftle(const DevGrid<T> &g, FieldPtrs<T> f, lcsdata_t *ftle, lcsdata_t Tint, dim3 blk, dim3 grd) {
    const int inc = opt_->incompressible;
    if (g.P.curv) {
      if (g.P.has_flags) k_ftle<T, lcsdata_t, true, true><<<grd, blk, 0, stream_>>>(g, f, ftle, Tint, inc);
      else k_ftle<T, lcsdata_t, false, true><<<grd, blk, 0, stream_>>>(g, f, ftle, Tint, inc);
    } else {
      if (g.P.has_flags) k_ftle<T, lcsdata_t, true><<<grd, blk, 0, stream_>>>(g, f, ftle, Tint, inc);
      else k_ftle<T, lcsdata_t, false><<<grd, blk, 0, stream_>>>(g, f, ftle, Tint, inc);
    }
  }

  bool launch_ftle(DiagT &d, std::string &msg) {
    const DevGrid<T> &g = dgrid(d);
    const dim3 blk(32, 8, 1), grd = node_grid(g);
    FieldPtrs<T> f{};
    for (int c = 0; c < 3; c++) f.f[c] = d.composed[c];
    counters_.kernel_launches++;
    launch_ftle(g, f, d.ftle, d.T_, blk, grd);
    CK(cudaGetLastError());
    return true;
  }

  // velocity snapshot of ring step `step` (write_flowmap_substep's u_np1 file, shared by
  // every diagnostic; steps 0 .. kMaxVelocitySteps-1 kept)
  static constexpr int kMaxVelocitySteps = 4096;
  bool snapshot_velocity(long step, std::string &msg) {
    if (step < 0 || step >= kMaxVelocitySteps) return true;
    if (vring_.empty()) {
      vring_.assign((size_t)3 * kMaxVelocitySteps, nullptr);
      vwritten_.assign(kMaxVelocitySteps, 0);
    }
    if (!vring_[3 * step])
      for (int c = 0; c < 3; c++)
        if (!(vring_[3 * step + c] = arena_.alloc<TV>(N_, msg))) return false;
    FieldPtrs<TV> u{};
    FieldPtrsW<TV> dst{};
    for (int c = 0; c < 3; c++) {
      u.f[c] = u_[cur_][c];
      dst.f[c] = vring_[3 * step + c];
    }
    k_vel_snapshot<T, TV><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, u, dst);
    counters_.kernel_launches++;
    CK(cudaGetLastError());
    vwritten_[step] = 1;
    return true;
  }

  // the velocity snapshots are kept when VELOCITY_IO or VELOCITY_INVARIANTS asks for them
  // (write_flowmap_substep, src/flowmap_m.f90:140); VELOCITY_IO matters only with files
  bool need_velocity_ring() const { return opt_->velocity_invariants || (opt_->write_lcs && opt_->write_velocity); }

  // The frame's output file (write_lcs / write_ftle, src/io_nohdf5_m.f90:47-264): name,
  // header, and the device blocks copied into pinned staging on the stream; the writer thread
  // formats and writes once the copies are done.
  bool enqueue_output(DiagT &d, long ustep, std::string &msg) {
    long long findex = (long long)fnint((double)(t_np1_ / d.h));
    if (d.type == FTLE_FWD) findex -= (long long)fnint((double)(d.T_ / d.h));
    std::string idx;
    if (!lcs_file_index(findex, idx)) {
      msg = "ERROR: unsupported range for file index, " + std::to_string(findex);
      return false;
    }
    if (!writer_) writer_.reset(new LcsWriter());
    OutputJob job;
    job.path = "./cfd2lcs_output/" + d.label + "_" + idx + ".dat";
    const long NN = dN(d);
    int nn[3];
    for (int a = 0; a < 3; a++) {
      nn[a] = d.lg ? d.lg->dg.P.n[a] : n_[a];
      job.n[a] = nn[a];
      job.lines[a] = d.lg ? d.lg->out_lines[a] : out_lines_[a];
      if (!d.lg) job.coords[a] = out_coords_[a];
    }
    job.flags = d.lg ? d.lg->out_flags : out_flags_;
    const std::string title = d.label + "-FTLE";
    std::string h = "TITLE = \"" + title + "\"\nVARIABLES =\n\"X\"\n\"Y\"\n\"Z\"\n";
    if (opt_->write_flowmap) h += "\"FM-X\"\n\"FM-Y\"\n\"FM-Z\"\n";
    if (opt_->write_velocity) h += "\"U-X\"\n\"U-Y\"\n\"U-Z\"\n";
    if (opt_->write_bcflag) h += "\"FLAG\"\n";
    if (opt_->velocity_invariants) h += "\"Q\"\n\"C\"\n\"D\"\n\"H\"\n\"L2\"\n";
    h += "\"FTLE\"\nZONE\nT = \"" + title + "\"\n";
    char tbuf[32], line[128];
    format_es((double)t_np1_, 18, 4, tbuf);
    tbuf[18] = 0;
    std::snprintf(line, sizeof(line), "STRANDID = %010d, SOLUTIONTIME = %s\n", 1, tbuf);
    h += line;
    std::snprintf(line, sizeof(line), "I = %010d J = %010d K = %010d\n", nn[0], nn[1], nn[2]);
    h += line;
    h += "ZONETYPE = Ordered, DATAPACKING = BLOCK\n";
    job.header = h;
    // blocks: X Y Z [FM] [U] [FLAG] [Q C D H L2] FTLE
    struct Src {
      const void *p;
      size_t esize;
    };
    std::vector<Src> staged;
    std::vector<OutputBlock> blocks;
    size_t bytes = 0;
    auto stage = [&](const void *p, size_t esize) {
      OutputBlock b;
      b.kind = esize == 8 ? OutputBlock::STAGED_F64 : OutputBlock::STAGED_F32;
      b.offset = bytes;
      bytes += ((size_t)NN * esize + 255) / 256 * 256;
      staged.push_back({p, esize});
      blocks.push_back(b);
    };
    auto plain = [&](OutputBlock::Kind k) {
      OutputBlock b;
      b.kind = k;
      blocks.push_back(b);
    };
    plain(OutputBlock::LINE_X);
    plain(OutputBlock::LINE_Y);
    plain(OutputBlock::LINE_Z);
    if (opt_->write_flowmap)
      for (int c = 0; c < 3; c++) stage(d.composed[c], sizeof(T));
    if (opt_->write_velocity) {
      // lp%ugrid: the frame's starting velocity when its snapshot exists, else zero (reset_lp)
      const bool have = ustep >= 0 && ustep < (long)vwritten_.size() && vwritten_[ustep];
      for (int c = 0; c < 3; c++) {
        if (d.lg) stage(d.lg->ugrid[c], sizeof(T));
        else if (have) stage(vring_[3 * ustep + c], sizeof(TV));
        else plain(OutputBlock::ZERO);
      }
    }
    if (opt_->write_bcflag) plain(OutputBlock::FLAG);
    if (opt_->velocity_invariants) {
      const int order[5] = {0, 2, 1, 3, 4};  // Q, C, D, H, L2 (the fields are kept Q, D, C, H, L2)
      for (int q : order) stage(d.inv[q], sizeof(lcsdata_t));
    }
    stage(d.ftle, sizeof(lcsdata_t));
    void *buf = nullptr;
    const int bi = writer_->acquire(std::max<size_t>(bytes, 1), &buf, msg);
    if (bi < 0) return false;
    size_t q = 0;
    for (OutputBlock &b : blocks) {
      if (b.kind != OutputBlock::STAGED_F64 && b.kind != OutputBlock::STAGED_F32) continue;
      CK(cudaMemcpyAsync(static_cast<char *>(buf) + b.offset, staged[q].p, (size_t)NN * staged[q].esize, cudaMemcpyDeviceToHost,
                         stream_));
      q++;
    }
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, stream_));
    job.blocks = std::move(blocks);
    job.ready = ev;
    job.buffer = bi;
    writer_->submit(std::move(job));
    return true;
  }

  // lp%ugrid of a refined diagnostic (reconstruct_flowmap, src/flowmap_m.f90:214-245): zero
  // (reset_lp) unless the snapshot of ring step ustep exists, else that snapshot padded with
  // its periodic images, fitted when the interpolator is a B-spline, and sampled at the nodes.
  bool make_ugrid(DiagT &d, long ustep, std::string &msg) {
    LcsGrid<T> &L = *d.lg;
    if (!L.ugrid[0])
      for (int c = 0; c < 3; c++)
        if (!(L.ugrid[c] = arena_.alloc<T>(L.N, msg))) return false;
    const bool have = ustep >= 0 && ustep < (long)vwritten_.size() && vwritten_[ustep];
    if (!have) {
      for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(L.ugrid[c], 0, L.N * sizeof(T), stream_));
      return true;
    }
    if (!upad_[0])
      for (int c = 0; c < 3; c++)
        if (!(upad_[c] = arena_.alloc<TV>(ntot_, msg)) || !(upcoef_[c] = arena_.alloc<TV>(ntot_, msg))) return false;
    FieldPtrs<TV> src{};
    FieldPtrsW<TV> dst{};
    for (int c = 0; c < 3; c++) {
      src.f[c] = vring_[3 * ustep + c];
      dst.f[c] = upad_[c];
    }
    k_pad_snapshot<T, TV><<<(unsigned)((ntot_ + 255) / 256), 256, 0, stream_>>>(dg_, src, dst, ntot_);
    counters_.kernel_launches++;
    const int interp = interpolator();
    const bool spline = interp == QUADRATIC || interp == CUBIC;
    VelFields<TV> V{};
    SplineAxes<T> sa{};
    for (int c = 0; c < 3; c++) V.un[c] = V.unp1[c] = upad_[c];
    if (spline) {
      const int deg = interp == QUADRATIC ? 2 : 3;
      if (!ensure_spline(deg, msg) || !fit(vsplines_[deg].axes, upad_, upcoef_, msg)) return false;
      for (int c = 0; c < 3; c++) V.cs[0][c] = upcoef_[c];
      sa = splines_[deg].axes;
    }
    FieldPtrsW<T> out{};
    for (int c = 0; c < 3; c++) out.f[c] = L.ugrid[c];
    const dim3 grd = node_grid(L.dg), blk(32, 8, 1);
    const int iv = interp_variant(interp, sa);
    if (iv == INTERP_NEAREST) k_sample_ugrid<T, TV, INTERP_NEAREST><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    else if (iv == INTERP_LINEAR) k_sample_ugrid<T, TV, INTERP_LINEAR><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    else if (iv == INTERP_TSE) k_sample_ugrid<T, TV, INTERP_TSE><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    else if (iv == INTERP_TSE_LIMIT) k_sample_ugrid<T, TV, INTERP_TSE_LIMIT><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    else if (iv == INTERP_SPLINE4) k_sample_ugrid<T, TV, INTERP_SPLINE4><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    else k_sample_ugrid<T, TV, INTERP_SPLINE><<<grd, blk, 0, stream_>>>(L.dg, dg_, sa, V, out);
    counters_.kernel_launches++;
    CK(cudaGetLastError());
    return true;
  }

  bool launch_invariants(DiagT &d, long ustep, std::string &msg) {
    if (!d.inv[0])
      for (int q = 0; q < 5; q++)
        if (!(d.inv[q] = arena_.alloc<lcsdata_t>(dN(d), msg))) return false;
    if (d.lg) {
      // the invariants of the lcs grid's lp%ugrid (gradient on the lcs grid)
      FieldPtrs<T> u{};
      for (int c = 0; c < 3; c++) u.f[c] = d.lg->ugrid[c];
      FieldPtrsW<T> o3{}, o2{};
      for (int q = 0; q < 3; q++) o3.f[q] = d.inv[q];
      o2.f[0] = d.inv[3];
      o2.f[1] = d.inv[4];
      k_invariants<T, T><<<node_grid(d.lg->dg), dim3(32, 8, 1), 0, stream_>>>(d.lg->dg, u, 1, o3, o2);
      counters_.kernel_launches++;
      CK(cudaGetLastError());
      return true;
    }
    const bool have = ustep >= 0 && ustep < (long)vwritten_.size() && vwritten_[ustep];
    FieldPtrs<TV> u{};
    for (int c = 0; c < 3; c++) u.f[c] = have ? vring_[3 * ustep + c] : nullptr;
    FieldPtrsW<T> o3{}, o2{};
    for (int q = 0; q < 3; q++) o3.f[q] = d.inv[q];
    o2.f[0] = d.inv[3];
    o2.f[1] = d.inv[4];
    if (dg_.P.curv) k_invariants<T, TV, true><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, u, have ? 1 : 0, o3, o2);
    else k_invariants<T, TV><<<node_grid(), dim3(32, 8, 1), 0, stream_>>>(dg_, u, have ? 1 : 0, o3, o2);
    counters_.kernel_launches++;
    CK(cudaGetLastError());
    return true;
  }

  void launch_reset(DiagT &d) {
    const dim3 blk(32, 8, 1);
    counters_.kernel_launches++;
    d.since_sort = 0;  // the particles are back on their nodes, in node order
    d.base_ms = -1;
    d.excess_ms = 0;
    if (d.lg) {
      FieldPtrs<T> pos{};
      for (int c = 0; c < 3; c++) pos.f[c] = d.lg->pos[c];
      k_reset_refined<T><<<node_grid(d.lg->dg), blk, 0, stream_>>>(d.lg->dg, pos, d.lg->nos_reset[0], d.lg->nos_reset[1], d.lg->nos_reset[2],
                                                                   d.P);
    } else {
      k_reset_particles<T><<<node_grid(), blk, 0, stream_>>>(dg_, d.P);
    }
  }

  // Re-sorts the particle slots by grid cell (32 x 4 x 2 tiles, x fastest) every kSortInterval
  // subcycles, so that the particles of a block gather neighbouring spline taps as the SL
  // kernel's blocks do.  Results do not depend on the order: every particle is advanced
  // independently and the snapshot reads it back through the inverse map.  Measured on B200
  // (ABC 256^3, RK3 CUBIC, FP64): every 6 / 4 / 3 / 2 subcycles gave 332.9 / 330.9 / 328.9 /
  // 326.0 ms per update (the forward launch 7.55 -> 6.94 ms against 0.9 ms per sort).
#ifndef CFD2LCS_SORT_INTERVAL
#define CFD2LCS_SORT_INTERVAL 2
#endif
  static constexpr int kSortInterval = CFD2LCS_SORT_INTERVAL;
  int sort_every_ = 0;  // CFD2LCS_B200_SORT_EVERY at cfd2lcs_init (0: the default below)
  int sort_interval(int interp) const { return sort_every_ > 0 ? sort_every_ : kSortInterval; }
  // Re-sort schedule of a set whose forward kernel gathers (not the staged family): a sort
  // restores the coalescing the launches lose as the particles drift from the order of the
  // last sort, so it pays once the time they have lost since that sort -- each launch's event
  // time minus the first launch's after the sort -- reaches the sort's own event time (the
  // rent-or-buy rule: at most twice the best fixed schedule's cost).  Launch times reach the
  // engine when an update is collected, so the rule acts on update boundaries; until a sort
  // has been timed the set re-sorts every kSortInterval subcycles.  Measured on B200, ABC
  // 256^3 RK2 LINEAR: fixed intervals of 2 / 6 / 24 subcycles gave 59.2 / 52.4 / 50.0 ms per
  // update (the launch 1.16 -> 1.20 -> 1.23 ms against 0.88 ms per sort), never re-sorting 51.2.
  // CFD2LCS_B200_SORT_EVERY=n fixes the interval at n subcycles instead.  The batched form's
  // instances keep the fixed interval: with other instances' kernels interleaved, a sort's event
  // span is not its cost (measured on the 64-instance batch: 89 ms per step with the rule, 81 ms
  // with the interval).
  bool sort_due(const DiagT &d) const {
    if (sort_every_ > 0) return d.since_sort >= sort_every_;
    if (d.sort_ms <= 0 || opt_->shared_device) return d.since_sort >= kSortInterval;
    return d.excess_ms >= d.sort_ms;
  }
  // fwd_tile: the 16 x 4 x 4-cell tiles the staged forward kernel reads, else the 32 x 4 x 2
  // tiles that suit the gathering kernel
  bool sort_particles(DiagT &d, std::string &msg, bool fwd_tile = false) {
    d.sort_geom = fwd_tile ? sort_tiles(n_, FWT_TX, FWT_TY, FWT_TZ) : sort_tiles(n_, 32, SORT_TY, SORT_TZ);
    if (!sort_slots(d.P, d.P2, d.pkey, d.pcnt, d.poffs, d.ptsum, (int)dN(d), d.sort_geom, msg)) return false;
    std::swap(d.P, d.P2);
    return true;
  }

  // counting sort of np particle slots of a by cell into b (tiles of geometry st)
  bool sort_slots(const Particles<T> &a, const Particles<T> &b, unsigned *key, int *cnt, int *offs, int *tsum, int np, const SortTiles &st,
                  std::string &msg) {
    const int blk = 256, grd = (np + blk - 1) / blk;
    const int ncell = (int)sort_key_space(st);
    const int ntile = (ncell + SORT_TILE - 1) / SORT_TILE;
    k_particle_count<T><<<grd, blk, 0, stream_>>>(dg_, a, key, cnt, np, st);
    k_scan_tiles<<<ntile, 256, 0, stream_>>>(cnt, offs, tsum, ncell);
    k_scan_tile_sums<<<1, 1024, 0, stream_>>>(tsum, ntile);
    k_particle_scatter<T><<<grd, blk, 0, stream_>>>(a, b, key, offs, tsum, np);
    CK(cudaGetLastError());
    counters_.kernel_launches += 4;
    return true;
  }

  const Options *opt_;
  int handle_count_ = 0;  // handles given out so far (a failed LP_TRACER injection uses one up)
  TV *upad_[3] = {nullptr, nullptr, nullptr}, *upcoef_[3] = {nullptr, nullptr, nullptr};  // refined lp%ugrid scratch
  std::unique_ptr<LcsWriter> writer_;  // created by the first output file
  std::shared_ptr<const std::vector<double>> out_lines_[3];
  std::shared_ptr<const std::vector<double>> out_coords_[3];  // non-rectilinear grids only
  std::shared_ptr<const std::vector<int8_t>> out_flags_;
  HostGrid<lcsdata_t> hg_;
  DevGrid<T> dg_{};
  DevArena arena_;
  cudaStream_t stream_ = nullptr;
  std::vector<cudaEvent_t> ev_;
  int n_[3] = {0, 0, 0};
  long N_ = 0, ntot_ = 0;
  TV *u_[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  TV *ucoef_[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int ucoef_deg_[2] = {0, 0};
  int cur_ = 0;
  lcsdata_t *stage_ = nullptr;
  DevReduce *red_ = nullptr, *red_host_ = nullptr;
  int red_err_ = 0;
  SplineSet<T> splines_[4];
  std::vector<TV *> vring_;     // velocity snapshots by ring step (VELOCITY_INVARIANTS)
  std::vector<char> vwritten_;
  SplineSet<TV> vsplines_[4];
  std::vector<DiagT> diags_;
  lcsdata_t t_n_ = 0, t_np1_ = 0;
  bool first_call_ = true;
  bool begun_ = false;
  Counters counters_;
  // event-timed spans of the update in flight: phase index 1..5, or one of the hot kernels
  enum { SPAN_SL = 100, SPAN_FWD = 101, SPAN_SORT = 102 };
  struct Span {
    cudaEvent_t a, b;
    int kind;
    int tune = -1;   // hot-kernel spans while the tuner samples: family * 2 + variant
    int diag = -1;   // forward launches and sorts of a set on the sort_due schedule: its index
    int since = 0;   // forward launches: subcycles since that set's last sort or reset
  };
  std::vector<cudaEvent_t> evpool_;
  size_t evnext_ = 0;
  std::vector<Span> spans_;

  // records the next pooled event on the stream (the pool grows to one update's needs)
  bool mark(cudaEvent_t &e, std::string &msg) {
    if (evnext_ == evpool_.size()) {
      cudaEvent_t x;
      CK(cudaEventCreate(&x));
      evpool_.push_back(x);
    }
    e = evpool_[evnext_++];
    CK(cudaEventRecord(e, stream_));
    return true;
  }
};

}  // namespace cfd2lcs
