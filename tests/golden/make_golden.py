"""Generates the golden fixtures of tests/test_golden_configs.py (TEST INFRASTRUCTURE).

Runs the oracle -- the plain-C restatement of libcfd2lcs's single-rank path, built from
oracle/cfd2lcs_oracle.c -- on the benchmark configurations over their full FTLE horizon and
stores, per diagnostic, the last frame's FTLE field (FP64, every point), the composed flow
map on every 16th point (FP64) and the reference's work counters.  The inputs are the
seeded synthetic flows of tests.workloads, regenerated identically by the test.

    python tests/golden/make_golden.py [dg512 abc48 turb48] [--threads N]

Cases (the reference's example drivers set the same options, examples/double_gyre_c.c:
301-339 and examples/abc_flow_c.c:295-333):
  dg512  : double gyre 512x256x1 (A=0.1, eps=0.25, omega=2pi/10), slip walls, backward FTLE,
           T=15, h=1.5, dt=0.1, RK2, LINEAR, 161 updates (t = 0 .. 16; last frame at t=15
           composes all 10 sub-flow maps).
  abc48  : ABC flow 48^3 periodic (A=sqrt3, B=sqrt2, C=1), forward and backward FTLE, T=10,
           h=1, dt=0.05, RK3, CUBIC, 201 updates (last frame at t=10, all 10 sub-maps).
  turb48 : the 64-mode |k|<=32 seeded turbulence (FP32 field values) at 48^3, backward FTLE,
           T=2, h=0.2, dt=0.01, RK2, LINEAR, 210 updates (last frame at t=2, 10 sub-maps).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from tests import workloads as W  # noqa: E402

FM_STRIDE = 16  # composed flow map stored on every 16th point (flat i-fastest index)

CASES = {
    "dg512": dict(kind="dg", n=(512, 256), dirs=(1,), T=15.0, h=1.5, dt=0.1, integrator=2, interpolator=1, updates=161),
    "abc48": dict(kind="abc", n=48, dirs=(0, 1), T=10.0, h=1.0, dt=0.05, integrator=3, interpolator=3, updates=201),
    "turb48": dict(kind="turb", n=48, dirs=(1,), T=2.0, h=0.2, dt=0.01, integrator=2, interpolator=1, updates=210),
}


def case_flow(c):
    """(grid, velocity(t) -> (u, v, w) FP64 Fortran-ordered arrays)."""
    if c["kind"] == "dg":
        g = W.double_gyre_grid(*c["n"])
        return g, (lambda t: W.double_gyre_velocity(g, t))
    if c["kind"] == "abc":
        g = W.abc_grid(c["n"])
        vel = W.abc_velocity(g)
        return g, (lambda t: vel)
    g = W.abc_grid(c["n"])
    modes = W.turbulence_modes()
    return g, (lambda t: tuple(a.astype(np.float64) for a in W.turbulence_velocity(g, t, modes)))


def run_case(api, c):
    """Drives `api` (oracle.Oracle or libcfd2lcs_b200.Cfd2lcs) through the case; returns the
    diagnostic handles."""
    g, vel = case_flow(c)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    handles = [api.diagnostic_init(d, 0, c["T"], c["h"], f"d{d}") for d in c["dirs"]]
    api.set_option("INTEGRATOR", c["integrator"])
    api.set_option("INTERPOLATOR", c["interpolator"])
    for k in range(c["updates"]):
        t = W.time_at(k, c["dt"])
        u, v, w = vel(t)
        api.update(u, v, w, t)
    return g, handles


def fm_sample(fm):
    """(3, ni, nj, nk) -> (3, m): every FM_STRIDE-th point in i-fastest order."""
    flat = np.stack([np.asarray(fm[c]).ravel(order="F") for c in range(3)])
    return flat[:, ::FM_STRIDE]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*", default=list(CASES))
    ap.add_argument("--threads", type=int, default=len(os.sched_getaffinity(0)))
    a = ap.parse_args()
    from oracle.oracle import Oracle
    o = Oracle("dp")
    for name in a.cases:
        c = CASES[name]
        o.reset()
        o.set_threads(a.threads)
        t0 = time.time()
        g, handles = run_case(o, c)
        assert o.error() == 0, o.error_msg()
        out = {"updates": np.int64(c["updates"]), "fm_stride": np.int64(FM_STRIDE)}
        for d, h in zip(c["dirs"], handles):
            out[f"ftle_{d}"] = np.asarray(o.ftle(h), dtype=np.float64).ravel(order="F")
            out[f"fm_{d}"] = fm_sample(o.flowmap(h)).astype(np.float64)
        for k in ("integrations_fwd", "integrations_bkwd", "nsub_fwd", "nsub_bkwd", "ftle_frames"):
            out[k] = np.int64(o.counter(k))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {time.time() - t0:.1f} s with {o.threads()} threads -> {path} "
              f"({os.path.getsize(path) / 1e6:.2f} MB), frames {int(out['ftle_frames'])}", flush=True)


if __name__ == "__main__":
    main()
