"""FTLE error of the mixed-precision form against the plain FP64 form on the same inputs.

    python -m tests.accuracy --n 128 --T 10 --h 1 --updates 201

Runs the ABC workload twice through the C ABI (plain FP64, then MIXED_PRECISION), each for the
same number of updates, and reports max / RMS differences of the FTLE fields and composed
flow maps of the last frame.  The FP64 form is the parity-tested path (within 1e-8 of the
oracle on the parity cases), so it stands in for the FP64 oracle at sizes the CPU oracle
cannot run.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np


def run(mixed: bool, n: int, T: float, h: float, dt: float, updates: int, integrator: int, interp: int, dirs=(1, 0)):
    import torch

    import libcfd2lcs_b200 as L
    from tests import workloads as W

    api = L.Cfd2lcs("dp")
    api.reset()
    if mixed:
        api.set_option("MIXED_PRECISION", 1)
    g = W.abc_grid(n)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    hs = [api.diagnostic_init(d, 0, T, h, f"d{d}") for d in dirs]
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    u, v, w = W.abc_velocity(g)
    dev = [torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda() for a in (u, v, w)]
    t0 = time.perf_counter()
    for k in range(updates):
        api.update_device(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), W.time_at(k, dt))
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    err, msg = api.error()
    if err:
        raise RuntimeError(msg)
    out = {d: (api.ftle(hh).copy(), api.flowmap(hh).copy()) for d, hh in zip(dirs, hs)}
    cnt = api.counters()
    api.reset()
    return out, el, cnt


def compare(n=64, T=2.0, h=1.0, dt=0.05, updates=None, integrator=3, interp=3):
    updates = updates or int(round(T / dt)) + 1
    ref, el64, c64 = run(False, n, T, h, dt, updates, integrator, interp)
    mix, el32, c32 = run(True, n, T, h, dt, updates, integrator, interp)
    res = {"config": f"ABC {n}^3, T={T}, h={h}, dt={dt}, {updates} updates, integrator {integrator}, interpolator {interp}",
           "fp64_s": el64, "mixed_s": el32, "slots_composed": c64["slots_composed"]}
    for d in ref:
        f64, m64 = ref[d]
        f32, m32 = mix[d]
        dfl = np.abs(f32 - f64)
        key = "fwd" if d == 0 else "bkwd"
        res[key] = {"ftle_max_err": float(dfl.max()), "ftle_rms_err": float(math.sqrt(float((dfl ** 2).mean()))),
                    "ftle_p9999_err": float(np.quantile(dfl, 0.9999)), "points_over_1e-4": int((dfl > 1e-4).sum()),
                    "points": int(dfl.size), "ftle_range": [float(f64.min()), float(f64.max())],
                    "fm_max_err": float(np.abs(m32 - m64).max()),
                    "fm_points_over_1e-3": int((np.abs(m32 - m64).reshape(3, -1).max(axis=0) > 1e-3).sum())}
    return res


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--T", type=float, default=2.0)
    ap.add_argument("--h", type=float, default=1.0)
    ap.add_argument("--dt", type=float, default=0.05)
    ap.add_argument("--updates", type=int, default=None)
    ap.add_argument("--integrator", type=int, default=3)
    ap.add_argument("--interp", type=int, default=3)
    a = ap.parse_args()
    print(json.dumps(compare(a.n, a.T, a.h, a.dt, a.updates, a.integrator, a.interp)))
