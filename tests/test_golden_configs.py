"""Parity at the benchmark configurations' own sizes and full FTLE horizons.

The golden fixtures (tests/golden/*.npz) hold the oracle's results -- the CPU restatement
of the reference's single-rank path -- for three configurations run over a whole horizon,
written by tests/golden/make_golden.py:
  dg512  : double gyre 512x256x1, backward, T=15, h=1.5, dt=0.1, RK2, LINEAR, 161 updates
  abc48  : ABC flow 48^3, forward and backward, T=10, h=1, dt=0.05, RK3, CUBIC, 201 updates
  turb48 : 64-mode |k|<=32 turbulence at 48^3, backward, T=2, h=0.2, dt=0.01, RK2, LINEAR,
           210 updates
The GPU test drives the library through its C ABI with the same seeded inputs and compares
the last frame: FTLE at every point within 1e-9 (LINEAR) / 1e-8 (CUBIC), the composed flow
map on every 16th point within 1e-10 of the domain length, and the reference's work
counters exactly.  The flow-map bound is wider than the 1e-12 L of the short parity cases
(test_gpu_parity.py): the device contracts multiply-adds into FMAs and the oracle does not,
and over a whole horizon the flow's stretching amplifies those last-bit differences by up to
exp(lambda T) -- measured on B200: ABC 48^3 forward 5.8e-11 (1e-11 L) after T = 10, while its
FTLE stays within 1e-8.  The CPU tests check the fixtures themselves.
"""
import os

import numpy as np
import pytest

from tests.golden.make_golden import CASES, FM_STRIDE, fm_sample, run_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FTLE_TOL = {1: 1e-9, 3: 1e-8}
FM_TOL_REL = 1e-10
COUNTERS = ("integrations_fwd", "integrations_bkwd", "ftle_frames")


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _npts(c):
    n = c["n"]
    return n[0] * n[1] if isinstance(n, tuple) else n ** 3


@pytest.mark.parametrize("name", list(CASES))
def test_fixture_matches_its_case(name):
    c, ref = CASES[name], _load(name)
    assert int(ref["updates"]) == c["updates"] and int(ref["fm_stride"]) == FM_STRIDE
    n = _npts(c)
    for d in c["dirs"]:
        ftle = ref[f"ftle_{d}"]
        assert ftle.shape == (n,) and np.all(np.isfinite(ftle))
        assert ref[f"fm_{d}"].shape == (3, (n + FM_STRIDE - 1) // FM_STRIDE)
        # a full-horizon frame: the field is not the zero map of an empty ring
        assert float(np.max(np.abs(ref[f"fm_{d}"]))) > 0.1
    # every h boundary after the first produced a frame
    assert int(ref["ftle_frames"]) >= len(c["dirs"]) * int(round(c["T"] / c["h"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_library_matches_golden(name):
    import libcfd2lcs_b200 as L
    c, ref = CASES[name], _load(name)
    gpu = L.Cfd2lcs("dp")
    gpu.reset()
    g, handles = run_case(gpu, c)
    err, msg = gpu.error()
    assert err == 0, msg
    span = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
    tol = FTLE_TOL[c["interpolator"]]
    errs = {}
    for d, h in zip(c["dirs"], handles):
        ftle = np.asarray(gpu.ftle(h), dtype=np.float64).ravel(order="F")
        fm = fm_sample(gpu.flowmap(h))
        errs[d] = (float(np.max(np.abs(ftle - ref[f"ftle_{d}"]))), float(np.max(np.abs(fm - ref[f"fm_{d}"]))))
    print(f"{name}: " + ", ".join(f"dir {d}: FTLE max-abs {a:.2e}, flow map max-abs {b:.2e}" for d, (a, b) in errs.items()))
    for d, (dft, dfm) in errs.items():
        assert dft <= tol, f"{name} dir {d}: FTLE max-abs {dft:.3e} > {tol:.0e} ({errs})"
        assert dfm <= FM_TOL_REL * span, f"{name} dir {d}: flow map max-abs {dfm:.3e} > {FM_TOL_REL * span:.3e} ({errs})"
    cg = gpu.counters()
    for k in COUNTERS:
        assert cg[k] == int(ref[k]), (k, cg[k], int(ref[k]))
    gpu.finalize()
