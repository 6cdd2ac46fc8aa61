"""Composition one sub-flow map at a time with the particles re-sorted by cell between sub-maps
(k_compose_step, the large-grid path; forced on small grids with CFD2LCS_B200_COMPOSE_SORT_MIN=0)
against the node-ordered composition (k_compose): the per-point arithmetic is the same, so the
composed maps and FTLE fields must be bitwise equal -- across interpolators, boundary flags, a
2-D grid and both directions.  The oracle parity of the composition is in test_gpu_parity.py
and test_golden_configs.py."""
import os

import numpy as np
import pytest

from tests import scenarios as SC

pytestmark = pytest.mark.gpu


def _run(case, integrator, interp, sorted_, dirs, n=None, steps=None):
    import libcfd2lcs_b200 as L
    os.environ["CFD2LCS_B200_COMPOSE_SORT_MIN"] = "0" if sorted_ else str(1 << 40)
    try:
        gpu = L.Cfd2lcs("dp")
        gpu.reset()
        _, hs = SC.run(gpu, case, dirs, integrator, interp, n=n, steps=steps)
    finally:
        os.environ.pop("CFD2LCS_B200_COMPOSE_SORT_MIN", None)
    err, msg = gpu.error()
    assert err == 0, msg
    out = [gpu.flowmap(h) for h in hs] + [gpu.ftle(h) for h in hs]
    c = gpu.counters()
    gpu.reset()
    return out, c


@pytest.mark.parametrize("case,integrator,interp,n,steps", [("abc", 3, 3, 20, 26), ("abc_unsteady", 2, 1, 16, 18), ("dg", 2, 1, 64, 40),
                                                          ("mixed_bc", 3, 3, None, 12), ("turb", 2, 5, None, 16)])
def test_sorted_composition_is_bitwise(case, integrator, interp, n, steps):
    a, ca = _run(case, integrator, interp, True, (SC.FTLE_BKWD, SC.FTLE_FWD), n, steps)
    b, cb = _run(case, integrator, interp, False, (SC.FTLE_BKWD, SC.FTLE_FWD), n, steps)
    assert ca["slots_composed"] == cb["slots_composed"] and ca["slots_composed"] > ca["ftle_frames"]
    for x, y in zip(a, b):
        assert np.array_equal(x, y), float(np.max(np.abs(x - y)))
