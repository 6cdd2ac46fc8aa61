"""The allocation-free entry point cfd2lcs_reconstruct_noalloc_c, called through the C ABI.

Some callers cannot allocate device memory when they want the FTLE field (a solver whose
memory pool owns the GPU, for instance).  The entry point recomputes the latest frame into
buffers the caller allocated beforehand; its only scratch is a fixed device array.  The test
checks its output against the regular entry points (cfd2lcs_get_ftle_c /
cfd2lcs_get_flowmap_c) on two calls in a row, with the parity tolerances of the other GPU
tests.  This file is collected last so a stop-at-first-failure run has run everything else.
"""
import numpy as np
import pytest

from tests import scenarios as SC
from tests import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,integrator,interp", [("dg", 2, 1), ("abc", 3, 3)])
def test_reconstruct_noalloc_matches_regular_entry_points(case, integrator, interp):
    import torch

    import libcfd2lcs_b200 as L

    torch.cuda.set_device(0)
    api = L.Cfd2lcs("dp")
    api.reset()
    g, handles = SC.run(api, case, (SC.FTLE_BKWD, SC.FTLE_FWD), integrator, interp, n=32 if case == "dg" else 12,
                        steps=20 if case == "dg" else 12)
    err, msg = api.error()
    assert err == 0, msg
    N = int(np.prod(g.n))
    for h in handles:
        ref_ftle = api.ftle(h)
        ref_fm = api.flowmap(h)
        # the caller owns the output buffers (allocated before the call)
        d_ftle = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        d_fm = torch.full((3 * N,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):
            d_ftle.fill_(float("nan"))
            d_fm.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = api.reconstruct_noalloc(h, d_ftle.data_ptr(), d_fm.data_ptr())
            assert rc == 0, api.error()
            ftle = d_ftle.cpu().numpy().reshape(g.n, order="F")
            fm = d_fm.cpu().numpy()
            fm = np.stack([fm[c * N:(c + 1) * N].reshape(g.n, order="F") for c in range(3)])
            L_dom = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
            assert np.max(np.abs(ftle - ref_ftle)) <= (1e-8 if interp >= 2 else 1e-9), call
            assert np.max(np.abs(fm - ref_fm)) <= 1e-12 * L_dom, call
    api.reset()


def test_reconstruct_noalloc_rejects_without_frame():
    import libcfd2lcs_b200 as L

    api = L.Cfd2lcs("dp")
    api.reset()
    g = W.abc_grid(8)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    h = api.diagnostic_init(SC.FTLE_BKWD, 0, 1.0, 0.5)
    assert api.error()[0] == 0
    assert api.reconstruct_noalloc(h, 0, 0) == 1
    err, msg = api.error()
    assert err == 1 and "no FTLE frame" in msg
    api.reset()


def test_reconstruct_noalloc_rejects_more_submaps_than_its_table():
    """A frame of 257 sub-flow maps (T/h = 257; exact binary times so that every slot is
    written) exceeds the fixed 256-entry table: rejected with an error, nothing written."""
    import libcfd2lcs_b200 as L
    from tests import workloads as W

    api = L.Cfd2lcs("dp")
    api.reset()
    g = W.abc_grid(8)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    h = api.diagnostic_init(SC.FTLE_BKWD, 0, 257 * 0.0625, 0.0625)
    vel = W.abc_velocity(g)
    for k in range(260):
        api.update(*vel, k * 0.0625)
    err, msg = api.error()
    assert err == 0, msg
    assert api.reconstruct_noalloc(h, 0, 0) == 1
    err, msg = api.error()
    assert err == 1 and "more than the maximum" in msg, msg
    api.reset()


def test_reconstruct_noalloc_rejects_refined_grids():
    import libcfd2lcs_b200 as L
    from tests import workloads as W

    api = L.Cfd2lcs("dp")
    api.reset()
    g = W.abc_grid(8)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    h = api.diagnostic_init(SC.FTLE_BKWD, 1, 0.2, 0.1)
    vel = W.abc_velocity(g)
    for k in range(6):
        api.update(*vel, k * 0.05)
    assert api.error()[0] == 0
    assert api.reconstruct_noalloc(h, 0, 0) == 1
    err, msg = api.error()
    assert err == 1 and "resolution" in msg, msg
    api.reset()


def test_reconstruct_noalloc_single_precision():
    """The single-precision library (lcsdata_t = float): same output as its regular entry
    points on two calls in a row."""
    import torch

    import libcfd2lcs_b200 as L

    torch.cuda.set_device(0)
    api = L.Cfd2lcs("sp")
    api.reset()
    g, handles = SC.run(api, "abc", (SC.FTLE_BKWD,), 3, 3, n=12, steps=12)
    err, msg = api.error()
    assert err == 0, msg
    N = int(np.prod(g.n))
    h = handles[0]
    ref_ftle, ref_fm = api.ftle(h), api.flowmap(h)
    d_ftle = torch.empty((N,), dtype=torch.float32, device="cuda")
    d_fm = torch.empty((3 * N,), dtype=torch.float32, device="cuda")
    L_dom = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
    for call in range(2):
        d_ftle.fill_(float("nan"))
        d_fm.fill_(float("nan"))
        torch.cuda.synchronize()
        assert api.reconstruct_noalloc(h, d_ftle.data_ptr(), d_fm.data_ptr()) == 0, api.error()
        ftle = d_ftle.cpu().numpy().reshape(g.n, order="F")
        fm = d_fm.cpu().numpy()
        fm = np.stack([fm[c * N:(c + 1) * N].reshape(g.n, order="F") for c in range(3)])
        assert np.max(np.abs(ftle - ref_ftle)) <= 3e-4, call
        assert np.max(np.abs(fm - ref_fm)) <= 2e-5 * L_dom, call
    api.reset()
