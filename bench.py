"""Benchmark of the libcfd2lcs_b200 hot path (one JSON line on rank 0).

Metric: grid-pt*RK-steps/s -- the reference's own integration counter
(integrations_fwd + integrations_bkwd, src/lp_motion_m.f90:120-121: particles x subcycles)
divided by the device time of the updates -- plus the FTLE-field time of an h boundary.

A step is one cfd2lcs_update of the workload (every diagnostic advances through all of
its CFL subcycles).  Default workload: the 3-D ABC flow on 256^3 (A=sqrt3, B=sqrt2, C=1),
dt = 0.05, forward and backward FTLE with T = 10, h = 1, RK3, cubic B-spline, plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload abc256|dg512] [--precision fp64|mixed]

With --gpus N > 1 (under torchrun) each rank runs an independent replica of the workload
(the single-field path has no halo exchange): weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt·RK-steps/s + FTLE-field ms, mixed vs FP64 plain at stated FTLE error"
UNIT = "grid-pt·RK-steps/s"

# Algorithmic HBM bytes per grid point (or particle) and launch of the two hot kernels,
# s = bytes per real.  Backward SL subcycle: read the velocity data and the previous flow map,
# write the new flow map; linear/nearest read both time levels (2 x 3s), the B-spline forms
# read one blended coefficient field per RK stage (stages x 3s).  Forward particle subcycle:
# read+write position, displacement (6s each way) and node (12 B each way) plus the velocity
# data as above.
STAGES = {0: 1, 1: 1, 2: 2, 3: 3, 4: 3}

# DRAM bytes per point of one launch (dram__bytes_read.sum + dram__bytes_write.sum) from ncu
# captures at 192^3 (ABC flow, 7077888 points), scaled to the benchmark grid by its point count:
# (kernel, precision, interpolator, integrator) -> (bytes per point, where the figure comes from)
MEASURED_TRAFFIC = {
    ("k_sl_subcycle", "fp64", 3, 3): ((877.944576e6 + 201.871872e6) / 7077888, "ncu capture 2026-12-03, ABC 192^3, scaled by points"),
    ("k_fwd_subcycle", "fp64", 3, 3): ((964.329472e6 + 459.971072e6) / 7077888, "ncu capture 2026-12-03, ABC 192^3, scaled by points"),
    ("k_sl_subcycle", "mixed", 3, 3): ((524.9e6 + 171.9e6) / 7077888, "ncu capture 2026-12-03, ABC 192^3, scaled by points"),
    ("k_fwd_subcycle", "mixed", 3, 3): ((693.8e6 + 393.1e6) / 7077888, "ncu capture 2026-12-03, ABC 192^3, scaled by points"),
    ("k_sl_subcycle", "fp64", 1, 2): (1957.404e9 * 0.352992e-3 / 7077888, "ncu capture 2026-12-03, ABC 192^3, scaled by points"),
}


def sl_bytes_per_point(s: int, interp: int, integrator: int, sv: int = None) -> int:
    """s: bytes of a flow-map value, sv: bytes of a velocity value (4 in the mixed form)."""
    sv = sv or s
    vel = 2 * 3 * sv if interp in (0, 1) else STAGES[integrator] * 3 * sv
    return vel + 3 * s + 3 * s


def fwd_bytes_per_particle(s: int, interp: int, integrator: int, sv: int = None) -> int:
    sv = sv or s
    vel = 2 * 3 * sv if interp in (0, 1) else STAGES[integrator] * 3 * sv
    return vel + 2 * (6 * s + 12)


# interpolated points per integration step (the B-spline samples of the velocity)
SAMPLES = {0: 1, 1: 1, 2: 2, 3: 3, 4: 4}


def spline_flops_per_sample(interp: int) -> int:
    """Algorithmic FP64 flops of one B-spline sample of a 3-component field: per component
    the tensor-product contraction K^3 + K^2 + K FMAs (2 flops each), plus the basis of the
    three axes, 3K(K-1)/2 flops each (de Boor recurrence).  K = 4 (CUBIC) or 3 (QUADRATIC)."""
    K = 4 if interp == 3 else 3
    return 3 * 2 * (K ** 3 + K ** 2 + K) + 3 * (3 * K * (K - 1) // 2)


def advect_flops_per_point(kernel: str, interp: int, integrator: int):
    """B-spline interpolators only (None otherwise): samples per point times the sample cost,
    plus 6 flops of Runge-Kutta arithmetic per stage.  The backward SL kernel samples every
    stage but the first (which starts on the node) and the flow map once; the forward kernel
    samples every stage."""
    if interp not in (2, 3):
        return None
    n = SAMPLES[integrator]
    samples = n  # SL: n - 1 velocity stages + 1 flow-map sample; forward: n velocity stages
    return samples * spline_flops_per_sample(interp) + 6 * n


WORKLOADS = {
    "abc256": dict(kind="abc", n=256, dt=0.05, T=10.0, h=1.0, integrator=3, interpolator=3, dirs=(0, 1), t0=0.95,
                   desc="ABC flow 256^3 periodic, dt=0.05, FTLE fwd+bkwd T=10 h=1, RK3, cubic B-spline"),
    # profiling case: same flow and options, one backward diagnostic, two ring slots, so a
    # capture holds about 1.5 GB on the device while every field is larger than L2
    "abcprof": dict(kind="abc", n=192, dt=0.05, T=2.0, h=1.0, integrator=3, interpolator=3, dirs=(1,), t0=0.95,
                    desc="ABC flow 192^3 periodic, dt=0.05, FTLE bkwd T=2 h=1, RK3, cubic B-spline (profiling case)"),
    "abcproffwd": dict(kind="abc", n=192, dt=0.05, T=2.0, h=1.0, integrator=3, interpolator=3, dirs=(0,), t0=0.95,
                       desc="ABC flow 192^3 periodic, dt=0.05, FTLE fwd T=2 h=1, RK3, cubic B-spline (profiling case)"),
    "abcproflinfwd": dict(kind="abc", n=192, dt=0.05, T=2.0, h=1.0, integrator=2, interpolator=1, dirs=(0,), t0=0.95,
                          desc="ABC flow 192^3 periodic, dt=0.05, FTLE fwd T=2 h=1, RK2, linear (profiling case)"),
    "abcproflin": dict(kind="abc", n=192, dt=0.05, T=2.0, h=1.0, integrator=2, interpolator=1, dirs=(1,), t0=0.95,
                       desc="ABC flow 192^3 periodic, dt=0.05, FTLE bkwd T=2 h=1, RK2, linear (profiling case)"),
    # profiling case for the FTLE-field phase: frames of 10 sub-flow maps after 22 updates
    "abcring": dict(kind="abc", n=128, dt=0.05, T=1.0, h=0.1, integrator=3, interpolator=3, dirs=(0, 1), t0=0.95,
                    desc="ABC flow 128^3 periodic, dt=0.05, FTLE fwd+bkwd T=1 h=0.1, RK3, cubic B-spline (profiling case)"),
    "abcring256": dict(kind="abc", n=256, dt=0.05, T=1.0, h=0.1, integrator=3, interpolator=3, dirs=(0, 1), t0=0.95,
                       desc="ABC flow 256^3 periodic, dt=0.05, FTLE fwd+bkwd T=1 h=0.1, RK3, cubic B-spline (FTLE-field case)"),
    "abc256lin": dict(kind="abc", n=256, dt=0.05, T=10.0, h=1.0, integrator=2, interpolator=1, dirs=(0, 1), t0=0.95,
                      desc="ABC flow 256^3 periodic, dt=0.05, FTLE fwd+bkwd T=10 h=1, RK2, linear"),
    "dg512": dict(kind="dg", n=512, dt=0.1, T=15.0, h=1.5, integrator=2, interpolator=1, dirs=(1,), t0=1.4,
                  desc="double gyre 512x256x1, dt=0.1, FTLE bkwd T=15 h=1.5, RK2, linear"),
    "turb512": dict(kind="turb", n=512, dt=0.01, T=2.0, h=0.2, integrator=2, interpolator=1, dirs=(1,), t0=0.19,
                    desc="synthetic periodic turbulence 512^3 (64 seeded Fourier modes, k^-5/3, FP32 field values), "
                         "dt=0.01, FTLE bkwd T=2 h=0.2, RK2, linear"),
}


def make_grid(w, n=None):
    """(grid, host velocity(t) -> 3 numpy arrays, steady?)"""
    from tests import workloads as W
    if w["kind"] == "abc":
        g = W.abc_grid(n or w["n"])
        vel = W.abc_velocity(g)
        return g, (lambda t: vel), True
    if w["kind"] == "turb":
        g = W.abc_grid(n or w["n"])
        modes = W.turbulence_modes()
        return g, (lambda t: tuple(a.astype(np.float64) for a in W.turbulence_velocity(g, t, modes))), False
    g = W.double_gyre_grid(n or w["n"], (n or w["n"]) // 2)
    return g, (lambda t: W.double_gyre_velocity(g, t)), False


def turbulence_on_device(n, t, dev, chunk=16):
    """The seeded turbulence field of workloads.turbulence_velocity evaluated on the GPU (the
    host form takes minutes at 512^3): FP32 field values, returned as FP64 tensors in
    i-fastest order."""
    import torch
    from tests import workloads as W
    modes = W.turbulence_modes()
    L = 2.0 * math.pi
    line = (torch.arange(n, device=dev, dtype=torch.float64) + 0.5) * (L / n)
    out = [torch.empty(n * n * n, device=dev, dtype=torch.float64) for _ in range(3)]
    Y, X = torch.meshgrid(line, line, indexing="ij")  # (j, i), i fastest
    for k0 in range(0, n, chunk):
        kk = line[k0:k0 + chunk]
        acc = [torch.zeros((kk.numel(), n, n), device=dev, dtype=torch.float64) for _ in range(3)]
        for m in range(len(modes.k)):
            kx, ky, kz = (float(v) for v in modes.k[m])
            c0 = float(modes.omega[m]) * t + float(modes.phase[m])
            arg = (kx * X + ky * Y)[None, :, :] + (kz * kk)[:, None, None] + c0
            c = torch.cos(arg)
            for a in range(3):
                acc[a].add_(c, alpha=float(modes.a[m, a]))
        for a in range(3):
            out[a][k0 * n * n:(k0 + kk.numel()) * n * n] = acc[a].float().double().reshape(-1)
    return out


HBM_FALLBACK_GBS = 6650.0  # an earlier copy-bandwidth measurement on this B200 pool, used when no measured file exists


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def fp64_fma_tflops(iters: int = 16384, reps: int = 5) -> float:
    """The device's FP64 FMA rate (TFLOP/s) from the bench-only micro-benchmark library
    (libcfd2lcs_b200_fp64probe.so: eight independent FMA chains per thread, eight 256-thread
    blocks per SM, best of `reps` launches)."""
    import ctypes
    from libcfd2lcs_b200.build import build_probe
    lib = ctypes.CDLL(build_probe())
    lib.cfd2lcs_b200_fp64_fma_rate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.cfd2lcs_b200_fp64_fma_rate.restype = ctypes.c_int
    out = np.zeros(1, dtype=np.float64)
    rc = lib.cfd2lcs_b200_fp64_fma_rate(int(iters), int(reps), out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError(f"fp64 FMA probe failed (CUDA error {rc})")
    return float(out[0])


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json, else the fallback."""
    v = measured_peaks().get("hbm_gbs")
    if v:
        return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return HBM_FALLBACK_GBS, "fallback (no MEASURED_PEAKS.json on this box): 6650 GB/s"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons), "samples": len(sm)}


def rank_max(x: float, world: int, device) -> float:
    """Maximum of a per-rank time over all ranks (the job's time is its slowest rank's)."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample(w, steps: int, threads: int | None = None, n: int | None = None):
    """The oracle (CPU restatement of the reference path) on a bounded sample of the
    workload: the same flow, options, dt, T and h on a coarser grid, one update per step.
    96^3 for the ABC flow: about 10 s of oracle work per update on 16 host cores."""
    from oracle.oracle import Oracle
    o = Oracle("dp")
    o.reset()
    # every usable host core unless told otherwise: a launcher's OMP_NUM_THREADS (torchrun sets
    # 1 for N > 1) must not turn the baseline into a single-thread one
    o.set_threads(threads or len(os.sched_getaffinity(0)))
    nsample = n or (96 if w["kind"] == "abc" else 128)
    g, vel, steady = make_grid(w, nsample)
    o.init(g.n, g.x, g.y, g.z, g.flag)
    for d in w["dirs"]:
        o.diagnostic_init(d, 0, w["T"], w["h"], f"d{d}")
    o.set_option("INTEGRATOR", w["integrator"])
    o.set_option("INTERPOLATOR", w["interpolator"])
    t = w["t0"]
    u, v, wv = vel(t)
    o.update(u, v, wv, t)  # first call: no advection
    before = o.counter("integrations_fwd") + o.counter("integrations_bkwd")
    t_start = time.perf_counter()
    for s in range(steps):
        t = w["t0"] + (s + 1) * w["dt"]
        u, v, wv = vel(t)
        o.update(u, v, wv, t)
    el = time.perf_counter() - t_start
    work = o.counter("integrations_fwd") + o.counter("integrations_bkwd") - before
    assert o.error() == 0, o.error_msg()
    sample = (f"oracle on {g.n[0]}x{g.n[1]}x{g.n[2]} ({w['desc'].split(',')[0]} coarsened), same dt/T/h/integrator/"
              f"interpolator, {steps} update(s), {work} grid-pt*RK-steps in {el:.2f} s")
    return work / el, o.threads(), sample, el


def run_reference(args, w):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    rate, threads, sample, el = cpu_sample(w, steps)
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": steps,
            "warmup": 0, "ms_per_step": 1000.0 * el / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": w["desc"], "sample": "coarsened grid, see cpu_baseline"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def full_frame_update(w) -> int:
    """Index of the update whose FTLE frame composes nint(T/h) sub-flow maps that each span a
    whole h interval: the first h boundary after t0, plus T."""
    b1 = (math.floor(w["t0"] / w["h"] + 1e-9) + 1) * w["h"]
    return int(round((b1 + w["T"] - w["t0"]) / w["dt"]))


def ftle_error(a, b):
    d = np.abs(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64)).ravel()
    return {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d))), "p99_99": float(np.quantile(d, 0.9999)),
            "points_above_1e-4": int(np.count_nonzero(d > 1e-4)), "points": int(d.size)}


def run_form(args, w, precision, local, world, rank, clocks=False, e2e=False, horizon=None):
    """One library instance of the workload in one precision form: W warm-up updates, K timed
    updates (inputs resident in HBM), optionally K end-to-end updates through cfd2lcs_update_c,
    optionally continued (untimed) to update `horizon`, whose frame's FTLE fields it returns."""
    import torch
    import libcfd2lcs_b200 as L
    api = L.Cfd2lcs("dp")
    api.reset()
    if precision == "mixed":
        api.set_option("MIXED_PRECISION", 1)
    g, vel, steady = make_grid(w, args.n)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    handles = [api.diagnostic_init(d, 0, w["T"], w["h"], f"d{d}") for d in w["dirs"]]
    api.set_option("INTEGRATOR", w["integrator"])
    api.set_option("INTERPOLATOR", w["interpolator"])
    err, msg = api.error()
    if err:
        raise RuntimeError(msg)
    N = int(np.prod(g.n))
    dev = torch.device("cuda", local)
    total = args.warmup + args.steps

    def dev_fields(t):
        if w["kind"] == "turb":
            return turbulence_on_device(g.n[0], t, dev)
        u, v, wv = vel(t)
        return [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev) for a in (u, v, wv)]

    # steady flows: one resident field; the turbulence is generated on the device before each
    # step (outside the library's event-timed update); others: every step's field resident
    lazy = w["kind"] == "turb"
    fields = [dev_fields(w["t0"])] if steady else ([] if lazy else [dev_fields(w["t0"] + s * w["dt"]) for s in range(total + 1)])

    def step(s):
        f = fields[0] if steady else (dev_fields(w["t0"] + s * w["dt"]) if lazy or s >= len(fields) else fields[s])
        api.update_device(f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), w["t0"] + s * w["dt"])

    step(0)  # first call (no advection)
    for s in range(1, args.warmup + 1):
        step(s)
    err, msg = api.error()
    if err:
        raise RuntimeError(msg)
    # --- timed region (inputs resident in HBM) ---
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    c0, p0, k0, s0 = api.counters(), api.phase_times_ms(), api.kernel_times(), api.staged_launches()
    sampler = ClockSampler(local) if clocks else None
    if sampler:
        sampler.__enter__()
    for s in range(args.warmup + 1, total + 1):
        step(s)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    if world > 1:
        torch.distributed.barrier()
    c1, p1, k1, s1 = api.counters(), api.phase_times_ms(), api.kernel_times(), api.staged_launches()
    err, msg = api.error()
    if err:
        raise RuntimeError(msg)
    work = (c1["integrations_fwd"] + c1["integrations_bkwd"]) - (c0["integrations_fwd"] + c0["integrations_bkwd"])
    ms = p1["update_total"] - p0["update_total"]
    ms_max = rank_max(ms, world, dev)
    out = dict(api=api, g=g, N=N, handles=handles, work=work, ms=ms, ms_max=ms_max, value=world * work / (ms_max / 1000.0),
               launches=c1["kernel_launches"] - c0["kernel_launches"], c0=c0, c1=c1, p0=p0, p1=p1, k0=k0, k1=k1,
               clocks=sampler.summary() if sampler else None, staged={k: s1[k] - s0[k] for k in s1}, tuning=api.tuning())
    nxt = total + 1
    if e2e:
        # --- end to end: host arrays through cfd2lcs_update_c, FTLE read back each step ---
        pin = []
        for s in range(args.steps):
            t = w["t0"] + (total + 1 + s) * w["dt"]
            arrs = []
            if lazy:
                for a in dev_fields(t):
                    tt = torch.empty(N, dtype=torch.float64, pin_memory=True)
                    tt.copy_(a)
                    arrs.append(tt)
                    del a
            else:
                u, v, wv = vel(t)
                for a in (u, v, wv):
                    tt = torch.empty(N, dtype=torch.float64, pin_memory=True)
                    tt.numpy()[:] = a.ravel(order="F")
                    arrs.append(tt)
            pin.append(arrs)
            if steady:
                break
        res = torch.empty(N, dtype=torch.float64, pin_memory=True)
        nint = np.ascontiguousarray(g.n, dtype=np.int32)
        ce0 = api.counters()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t_e0 = time.perf_counter()
        for s in range(args.steps):
            arrs = pin[0] if steady else pin[s]
            tt = w["t0"] + (total + 1 + s) * w["dt"]
            api.lib.cfd2lcs_update_c(api._p(nint), arrs[0].data_ptr(), arrs[1].data_ptr(), arrs[2].data_ptr(), api.R(tt))
            for h in handles:
                api.lib.cfd2lcs_get_ftle_c(int(h), res.data_ptr())
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t_e0
        e2e_max = rank_max(e2e_s, world, dev)
        if world > 1:
            torch.distributed.barrier()
        ce1 = api.counters()
        err, msg = api.error()
        if err:
            raise RuntimeError(msg)
        e2e_work = (ce1["integrations_fwd"] + ce1["integrations_bkwd"]) - (ce0["integrations_fwd"] + ce0["integrations_bkwd"])
        out["e2e"] = {"value": world * e2e_work / e2e_max, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8,
                      "d2h_bytes_per_step": len(handles) * N * 8}
        nxt = total + 1 + args.steps
    if horizon is not None:
        if not steady:
            fields.clear()
        for s in range(nxt, horizon):
            step(s)
        # the update that ends the horizon: its frames compose every ring slot
        torch.cuda.synchronize()
        ph0, cf0 = api.phase_times_ms(), api.counters()
        step(horizon)
        torch.cuda.synchronize()
        ph1, cf1 = api.phase_times_ms(), api.counters()
        err, msg = api.error()
        if err:
            raise RuntimeError(msg)
        nfr = cf1["ftle_frames"] - cf0["ftle_frames"]
        if nfr > 0:
            out["full_frame"] = {"frames": nfr, "slots_composed_per_frame": (cf1["slots_composed"] - cf0["slots_composed"]) / nfr,
                                 **{k: (ph1[k] - ph0[k]) / nfr for k in ("snapshot", "compose", "ftle")}}
        out["ftle"] = {d: np.array(api.ftle(h), copy=True) for d, h in zip(w["dirs"], handles)}
        out["horizon_t"] = w["t0"] + horizon * w["dt"]
    return out


def hot_kernel_rooflines(r, w, precision, hbm, fp64_peak, hbm_src=None):
    """Roofline of the two hot kernels from one form's timed region: algorithmic bytes per
    launch over the CUDA-event launch time, against the measured HBM copy bandwidth."""
    N = r["N"]
    s_bytes = 8
    v_bytes = 8 if precision == "fp64" else 4
    k0, k1 = r["k0"], r["k1"]
    cands = []
    nsl, nfw = k1["sl_launches"] - k0["sl_launches"], k1["fwd_launches"] - k0["fwd_launches"]
    # the kernels that ran in the timed region (staged, gathering, or both while the tuner sampled)
    def kname(staged, n, st, ga):
        return st if staged == n else (ga if staged == 0 else st + "+" + ga)
    stl = "k_sl_tile"
    if w["interpolator"] == 1:
        # the staged LINEAR kernel: planes marching along z where the fields have tensor maps
        stl = "k_sl_march_lin" if r["staged"].get("sl_march", 0) == r["staged"]["sl"] > 0 else "k_sl_tile_lin"
    if nsl > 0:
        cands.append((kname(r["staged"]["sl"], nsl, stl, "k_sl_subcycle"), k1["sl_ms"] - k0["sl_ms"], nsl,
                      sl_bytes_per_point(s_bytes, w["interpolator"], w["integrator"], v_bytes)))
    if nfw > 0:
        cands.append((kname(r["staged"]["fwd"], nfw, "k_fwd_tile", "k_fwd_subcycle"), k1["fwd_ms"] - k0["fwd_ms"], nfw,
                      fwd_bytes_per_particle(s_bytes, w["interpolator"], w["integrator"], v_bytes)))
    rooflines = {}
    for name, tot_ms, nl, bpp in cands:
        avg_s = tot_ms / nl / 1000.0
        achieved = N * bpp / avg_s / 1e9
        rooflines[name] = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                           "frac": achieved / hbm if hbm else None, "peak_source": hbm_src,
                           "avg_launch_ms": avg_s * 1000.0, "share_of_step": tot_ms / r["ms"] if r["ms"] else None,
                           "algorithmic_bytes_per_point": bpp, "algorithmic_bytes_per_launch": N * bpp, "traffic": None}
        tpp = MEASURED_TRAFFIC.get((name, precision, w["interpolator"], w["integrator"]))
        if tpp is not None and w["kind"] == "abc":
            rooflines[name]["traffic"] = tpp[0] * N
            rooflines[name]["traffic_source"] = tpp[1]
        fpp = advect_flops_per_point(name, w["interpolator"], w["integrator"])
        if fpp is not None and fp64_peak:
            tf = N * fpp / avg_s / 1e12
            rooflines[name]["fp64"] = {"achieved": tf, "peak": fp64_peak, "unit": "TFLOP/s", "frac": tf / fp64_peak,
                                       "flops_per_point": fpp,
                                       "peak_source": "FMA micro-benchmark (libcfd2lcs_b200_fp64probe.so), this run"}
    return rooflines


def ftle_field_roofline(r, w, hbm, hbm_src=None):
    """FTLE-field time per frame (ring snapshot + composition + FTLE, CUDA events on the
    library's stream) against its HBM bound: per point nslot sub-map reads (3 FP64 each), the
    composed map (3) and the FTLE (1) -- (nslot*24 + 24 + 8) bytes.  Measured at the frame that
    ends the full horizon (every ring slot composed) when the run reached it, else averaged
    over the frames seen so far (rings still filling)."""
    nslot = int(round(w["T"] / w["h"]))
    ff = r.get("full_frame")
    if ff:
        ms, parts, frames, where = ff["snapshot"] + ff["compose"] + ff["ftle"], ff, ff["frames"], "full-horizon frame"
        slots = ff["slots_composed_per_frame"]
    else:
        p1, c1 = r["p1"], r["c1"]
        frames = c1["ftle_frames"]
        if not frames:
            return None
        parts = {k: p1[k] / frames for k in ("snapshot", "compose", "ftle")}
        ms, where, slots = sum(parts.values()), "average over the frames so far (rings filling)", c1["slots_composed"] / frames
    byts = r["N"] * (slots * 24 + 24 + 8)
    ach = byts / (ms / 1000.0) / 1e9
    return {"ms_per_frame": ms, "snapshot_ms": parts["snapshot"], "compose_ms": parts["compose"], "ftle_ms": parts["ftle"],
            "frames": frames, "slots_composed_per_frame": slots, "measured_at": where, "nslot": nslot, "algorithmic_bytes": byts,
            "bound_ms": byts / (hbm * 1e9) * 1e3 if hbm else None, "achieved_gbs": ach, "frac": ach / hbm if hbm else None,
            "peak_source": hbm_src}


def run_b200(args, w):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    import libcfd2lcs_b200 as L  # noqa: F401
    dev = torch.device("cuda", local)
    # the mixed form beside the plain FP64 one: same run, same workload, FTLE error over the
    # workload's full horizon (the ABC flow: 201 updates at 256^3)
    with_mixed = args.precision == "fp64" and args.mixed == "on" or (args.mixed == "auto" and args.precision == "fp64"
                                                                      and w["kind"] == "abc" and world == 1)
    horizon = full_frame_update(w) if (with_mixed or args.full_frame) else None
    r = run_form(args, w, args.precision, local, world, rank, clocks=True, e2e=True, horizon=horizon)
    api = r["api"]
    fp64_peak = fp64_fma_tflops() if w["interpolator"] in (2, 3) and args.precision == "fp64" else None
    hbm, hbm_src = hbm_peak()
    rooflines = hot_kernel_rooflines(r, w, args.precision, hbm, fp64_peak, hbm_src)
    roof = max(rooflines.values(), key=lambda x: x["share_of_step"] or 0) if rooflines else None
    c1, p0, p1 = r["c1"], r["p0"], r["p1"]
    frames = c1["ftle_frames"]
    ffr = ftle_field_roofline(r, w, hbm, hbm_src)
    g = r["g"]
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_max"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64 positions, f32 velocity", "data": "synthetic",
            "config": {"workload": w["desc"], "grid": list(g.n), "precision": args.precision, "l2": "inputs larger than L2 (126 MB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "ftle_field_ms": ffr["ms_per_frame"] if ffr else None, "ftle_field": ffr, "ftle_frames_seen": frames,
            "slots_composed_per_frame": (c1["slots_composed"] / frames if frames else None),
            "nsub_per_update": {"fwd": c1["nsub_fwd"], "bkwd": c1["nsub_bkwd"]},
            "gpu_launches": r["launches"], "staged_launches": r["staged"], "tuning": r["tuning"], "e2e": r["e2e"], "roofline": roof,
            "rooflines": rooflines,
            "phase_ms_per_step": {k: (p1[k] - p0[k]) / args.steps for k in p1}}
    if args.precision == "fp64":
        line["ftle_error"] = {"form": "plain FP64", "vs": "FP64 oracle (CPU restatement of the reference)",
                              "max_abs_tolerance": 1e-8 if w["interpolator"] >= 2 else 1e-9,
                              "where": "tests/test_golden_configs.py (benchmark configurations at 48^3 / 512x256 over their "
                                       "full horizon) and tests/test_gpu_parity.py (every integrator / interpolator)"}
    line["clocks"] = r["clocks"] if rank == 0 else None
    ftle64 = r.get("ftle")
    api.finalize()
    del r, api
    if with_mixed:
        m = run_form(args, w, "mixed", local, world, rank, horizon=horizon)
        mixed_ftle = m["ftle"]
        mroof = hot_kernel_rooflines(m, w, "mixed", hbm, None, hbm_src)
        line["mixed"] = {
            "form": "mixed: FP32 velocity levels, spline coefficients and stage blends; FP64 positions, flow maps, "
                    "composition, Cauchy-Green and eigen-solve",
            "value": m["value"], "unit": UNIT, "ms_per_step": m["ms_max"] / args.steps, "ratio_vs_fp64": m["value"] / line["value"],
            "ftle_field": ftle_field_roofline(m, w, hbm, hbm_src), "rooflines": mroof, "tuning": m["tuning"],
            "phase_ms_per_step": {k: (m["p1"][k] - m["p0"][k]) / args.steps for k in m["p1"]},
            "ftle_error": {"vs": "plain FP64 GPU path of this run (itself parity-tested against the FP64 oracle)",
                           "grid": list(g.n), "updates": horizon, "frame_t": m["horizon_t"],
                           **{("fwd" if d == 0 else "bkwd"): ftle_error(mixed_ftle[d], ftle64[d]) for d in w["dirs"]}}}
        m["api"].finalize()
        del m
    if args.precision == "mixed" and w["kind"] == "abc" and args.acc_n > 0 and rank == 0:
        # FTLE error of the mixed form against the plain FP64 path on the same flow and options
        # at a smaller grid, full T
        from tests import accuracy as A
        acc = A.compare(args.acc_n, w["T"], w["h"], w["dt"], None, w["integrator"], w["interpolator"])
        line["ftle_error"] = {"form": "mixed (FP32 velocity data, FP64 positions / flow maps / FTLE)",
                              "vs": "plain FP64 GPU path", "case": acc["config"],
                              **{d: acc[d] for d in ("fwd", "bkwd") if d in acc}}
    if rank == 0:
        if world == 1 and not args.no_cpu:
            rate, threads, sample, _ = cpu_sample(w, 1)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
            # the per-rank work of the reference: one thread, on a smaller sample of the workload
            rate1, _, sample1, _ = cpu_sample(w, 1, threads=1, n=48 if w["kind"] == "abc" else 64)
            line["cpu_baseline"]["single_thread"] = {"value": rate1, "unit": UNIT, "cores": 1, "sample": sample1}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


BATCH_DESC = ("batch of 64 independent instances: 32 double gyres 64x32..1024x512 (eps~U(.1,.3), A~U(.05,.15), dt=0.1) and "
              "32 ABC flows n^3, n in [32,192] (A,B,C~U(.5,2), dt=0.05); T~U(2,15), h=T/10, forward or backward per instance; "
              "RK2, linear; seed 64")


def batch_specs(seed: int = 64):
    """The 64 instances of the batched workload, drawn from one seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(32):
        nx = int(np.clip(round(2.0 ** rng.uniform(6.0, 10.0) / 32.0) * 32, 64, 1024))
        specs.append(dict(kind="dg", n=(nx, nx // 2), eps=float(rng.uniform(0.1, 0.3)), A=float(rng.uniform(0.05, 0.15)),
                          T=float(rng.uniform(2.0, 15.0)), dir=int(rng.integers(0, 2)), dt=0.1))
    for _ in range(32):
        n = int(rng.integers(2, 13)) * 16
        specs.append(dict(kind="abc", n=n, A=float(rng.uniform(0.5, 2.0)), B=float(rng.uniform(0.5, 2.0)),
                          C=float(rng.uniform(0.5, 2.0)), T=float(rng.uniform(2.0, 15.0)), dir=int(rng.integers(0, 2)), dt=0.05))
    return specs


def run_batch(args):
    """The batched form: every instance of this rank advanced by one cfd2lcs_batch_update_device_c
    per step (instances are dealt round-robin over ranks: strong scaling of a fixed batch).
    Time = wall clock of the batch calls with the device synchronised on both sides (the calls
    span one stream per instance); the same instances advanced one call per instance give the
    unbatched comparison."""
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    import libcfd2lcs_b200 as L
    from tests import workloads as W
    dev = torch.device("cuda", local)
    b = L.Batch("dp")
    b.reset()
    specs = [sp for i, sp in enumerate(batch_specs()) if i % world == rank]
    ids, vels, npts = [], [], []
    for sp in specs:
        if sp["kind"] == "dg":
            g = W.double_gyre_grid(*sp["n"])
            vel = (lambda g, sp: lambda t: W.double_gyre_velocity(g, t, A=sp["A"], eps=sp["eps"]))(g, sp)
        else:
            g = W.abc_grid(sp["n"])
            steady = W.abc_velocity(g, A=sp["A"], B=sp["B"], Cc=sp["C"])
            steady_dev = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev) for a in steady]
            vel = (lambda f: lambda t: f)(steady_dev)
        i = b.add(g.n, g.x, g.y, g.z, g.flag, 2, 1, 0.5, args.precision == "mixed")
        if i < 0 or b.diagnostic_init(i, sp["dir"], sp["T"], sp["T"] / 10.0) < 0:
            raise RuntimeError(b.error()[1])
        ids.append(i)
        vels.append(vel)
        npts.append(int(np.prod(g.n)))

    def fields(s):
        out = []
        for sp, vel in zip(specs, vels):
            f = vel(s * sp["dt"])
            if isinstance(f, tuple):
                f = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev) for a in f]
            out.append(f)
        return out

    def counters():
        return sum(b.counters(i)["integrations_fwd"] + b.counters(i)["integrations_bkwd"] for i in ids)

    def advance(s, together):
        f = fields(s)
        times = [s * sp["dt"] for sp in specs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if together:
            rc = b.update_device(ids, [x[0].data_ptr() for x in f], [x[1].data_ptr() for x in f], [x[2].data_ptr() for x in f], times)
        else:
            rc = 0
            for q, i in enumerate(ids):
                rc |= b.update_device([i], [f[q][0].data_ptr()], [f[q][1].data_ptr()], [f[q][2].data_ptr()], [times[q]])
        torch.cuda.synchronize()
        if rc:
            raise RuntimeError(b.error()[1])
        return time.perf_counter() - t0

    s = 0
    for _ in range(args.warmup + 1):
        advance(s, True)
        s += 1
    w0 = counters()
    el = 0.0
    for _ in range(args.steps):
        el += advance(s, True)
        s += 1
    work = counters() - w0
    w1 = counters()
    el_seq = 0.0
    for _ in range(args.steps):
        el_seq += advance(s, False)
        s += 1
    work_seq = counters() - w1
    el_max = rank_max(el, world, dev)
    el_seq_max = rank_max(el_seq, world, dev)
    tot = torch.tensor([float(work), float(work_seq), float(sum(npts))], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(tot)
    line = {"metric": METRIC, "value": float(tot[0]) / el_max, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * el_max / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64 positions, f32 velocity", "data": "synthetic",
            "config": {"workload": BATCH_DESC, "instances": 64, "points": int(tot[2]), "precision": args.precision,
                       "timing": "wall clock of the batch calls, device synchronised on both sides",
                       "parallelism": f"instances dealt over {world} GPUs" if world > 1 else "single GPU"},
            "unbatched": {"value": float(tot[1]) / el_seq_max, "unit": UNIT,
                          "what": "the same instances, one cfd2lcs_batch_update_device_c call per instance per step"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.reset()
    if world > 1:
        torch.distributed.destroy_process_group()


FD_EPS = 1e-6  # central-difference step of the adjoint check (velocity units)

ADJ_DESC = ("adjoint: J = mean backward FTLE over [pi/2,3pi/2]^3 of ABC flow on a 128^3 grid, 201 velocity levels "
            "(steady ABC + N(0, 0.01^2) noise from torch's CUDA generator, seed 7), 200 updates at dt=0.05, RK2, linear, "
            "flow-map checkpoint every 20 updates")


def run_adjoint(args):
    """The adjoint workload: one gradient dJ/du of every level (FP32, the sp library) timed by
    wall clock around the call (device synchronised on both sides); checked against the FP64
    gradient (dp library) and against central finite differences of the FP64 objective along
    random directions."""
    import torch
    world, rank, local = dist_setup()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    import libcfd2lcs_b200 as L
    from tests import workloads as W
    n = args.n or 128
    nl, dt, K = 201, 0.05, 20
    g = W.abc_grid(n)
    base = W.abc_velocity(g)
    gen7 = torch.Generator(device="cuda")
    gen7.manual_seed(7)
    b64 = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda() for a in base]
    lev64 = [[], [], []]
    for _ in range(nl):
        for c in range(3):
            lev64[c].append(b64[c] + 0.01 * torch.randn(b64[c].numel(), generator=gen7, device="cuda", dtype=torch.float64))
    times = [k * dt for k in range(nl)]
    x, y, z = g.x, g.y, g.z
    box = (x > 0.5 * math.pi) & (x < 1.5 * math.pi) & (y > 0.5 * math.pi) & (y < 1.5 * math.pi) & (z > 0.5 * math.pi) & (z < 1.5 * math.pi)
    w64 = torch.from_numpy(np.ascontiguousarray((box / box.sum()).astype(np.float64).ravel(order="F"))).cuda()
    lev32 = [[t.float() for t in comp] for comp in lev64]
    w32 = w64.float()
    # FP32 gradient (timed), after one untimed call
    L.adjoint_ftle(g, *lev32, times, w32, checkpoint_every=K, precision="sp", interpolator=args.adj_interp)
    runs = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J32, g32u, g32v, g32w = L.adjoint_ftle(g, *lev32, times, w32, checkpoint_every=K, precision="sp", interpolator=args.adj_interp)
        torch.cuda.synchronize()
        runs.append(time.perf_counter() - t0)
    el = min(runs)
    # FP64 gradient and finite differences
    J64, gu, gv, gw = L.adjoint_ftle(g, *lev64, times, w64, checkpoint_every=K, precision="dp", interpolator=args.adj_interp)
    num = sum(float(torch.sum((a.double() - b) ** 2)) for A, B in ((g32u, gu), (g32v, gv), (g32w, gw)) for a, b in zip(A, B))
    den = sum(float(torch.sum(b ** 2)) for B in (gu, gv, gw) for b in B)
    rel32 = math.sqrt(num / den) if den > 0 else None
    nfd = args.fd_dirs
    fd_err, fd_abs, fd_ad, fd_refined, tl_err = [], [], [], [], []
    gen = torch.Generator(device="cuda")
    gen.manual_seed(16)

    def central(d, eps):
        Jp, *_ = L.adjoint_ftle(g, *[[lev64[c][k] + eps * d[c][k] for k in range(nl)] for c in range(3)], times, w64,
                                checkpoint_every=K, precision="dp", gradient=False, interpolator=args.adj_interp)
        Jm, *_ = L.adjoint_ftle(g, *[[lev64[c][k] - eps * d[c][k] for k in range(nl)] for c in range(3)], times, w64,
                                checkpoint_every=K, precision="dp", gradient=False, interpolator=args.adj_interp)
        return (Jp - Jm) / (2 * eps)

    for q in range(nfd):
        d = [[torch.randn(lev64[c][k].numel(), generator=gen, device="cuda", dtype=torch.float64) for k in range(nl)] for c in range(3)]
        ad = sum(float(torch.dot(G[k], d[c][k])) for c, G in enumerate((gu, gv, gw)) for k in range(nl))
        _, tl = L.tangent_ftle(g, *lev64, times, w64, *d, precision="dp", interpolator=args.adj_interp)
        tl_err.append(abs(tl - ad) / max(abs(tl), abs(ad), 1e-300))
        fd = central(d, FD_EPS)
        fd_ad.append(ad)
        fd_abs.append(abs(fd - ad))
        err = abs(fd - ad) / max(abs(fd), abs(ad), 1e-300)
        fd_err.append(err)
        if err > 1e-3:
            # a direction whose directional derivative is small: the objective's FP64
            # rounding noise over 2 eps (grows as eps shrinks) and stencil-edge kinks inside
            # [-eps, eps] (grow with eps) are both visible; the sweep shows which
            ref = [{"eps": FD_EPS, "rel_err": err, "fd": fd}]
            for e in (FD_EPS * 10, FD_EPS / 10):
                f = central(d, e)
                ref.append({"eps": e, "rel_err": abs(f - ad) / max(abs(f), abs(ad), 1e-300), "fd": f})
            fd_refined.append({"direction": q, "adjoint": ad, "steps": ref})
    rms_ad = math.sqrt(sum(a * a for a in fd_ad) / len(fd_ad)) if fd_ad else 0.0
    # work: grid points x subcycles of the forward map, run twice (forward + segment recompute)
    api = L.Cfd2lcs("sp")
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    api.diagnostic_init(1, 0, times[-1], times[-1], "b")
    api.set_option("INTEGRATOR", 2)
    api.set_option("INTERPOLATOR", args.adj_interp)
    for k in range(nl):
        api.update_device(lev32[0][k].data_ptr(), lev32[1][k].data_ptr(), lev32[2][k].data_ptr(), times[k])
    work = api.counters()["integrations_bkwd"]
    api.reset()
    line = {"metric": METRIC, "value": work / el, "unit": UNIT, "n_gpus": 1, "steps": len(runs), "warmup": 1,
            "ms_per_step": 1000.0 * el, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": ADJ_DESC, "grid": [n, n, n], "levels": nl,
                                            "interpolator": "CUBIC" if args.adj_interp == 3 else "LINEAR",
                                            "timing": "wall clock of one gradient call (forward, checkpoints, reverse sweep), best of steps",
                                            "value_counts": "grid points x subcycles of the forward map per gradient"},
            "gradient_s": el, "J_fp32": J32, "J_fp64": J64,
            "gradient_fp32_vs_fp64_rel_l2": rel32,
            "tangent_linear_check": {"directions": nfd, "form": "FP64 forward-mode sweep vs FP64 adjoint, same directions",
                                     "max_rel_err": max(tl_err) if tl_err else None, "rel_errs": tl_err},
            "finite_difference_check": {"directions": nfd, "eps": FD_EPS, "form": "FP64 objective, central differences",
                                        "max_rel_err": max(fd_err) if fd_err else None,
                                        "median_rel_err": float(np.median(fd_err)) if fd_err else None, "rel_errs": fd_err,
                                        "max_abs_err_over_rms_derivative": max(fd_abs) / rms_ad if fd_abs and rms_ad > 0 else None,
                                        "adjoint_directional": fd_ad, "outliers_refined": fd_refined,
                                        "note": "relative errors above 1e-3 come from directions whose derivative is near zero "
                                                "(random cancellation); there the objective's FP64 rounding noise over 2 eps "
                                                "and trilinear stencil-edge kinks dominate, so the error is also given over "
                                                "the RMS directional derivative"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="abc256", choices=sorted(WORKLOADS) + ["batch64", "adj128"])
    ap.add_argument("--fd-dirs", type=int, default=16, help="adj128: finite-difference directions")
    ap.add_argument("--adj-interp", type=int, default=1, choices=(1, 3), help="adj128: LINEAR (1, the ADJ config) or CUBIC (3)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--acc-n", type=int, default=64, help="--precision mixed: grid of its FTLE error run (0: skip)")
    ap.add_argument("--mixed", default="auto", choices=["auto", "on", "off"],
                    help="also time the mixed form and state its FTLE error against this run's FP64 path over the full horizon "
                         "(auto: the ABC workloads on one GPU)")
    ap.add_argument("--n", type=int, default=None, help="override the grid size (smaller smoke runs)")
    ap.add_argument("--full-frame", action="store_true", help="run on to the full-horizon frame and time its FTLE field")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.workload == "adj128":
        if args.impl == "reference":
            world, rank, _ = dist_setup()
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint"}))
            return
        run_adjoint(args)
        return
    if args.workload == "batch64":
        if args.impl == "reference":
            world, rank, _ = dist_setup()
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched form (one instance per process)"}))
            return
        run_batch(args)
        return
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()
