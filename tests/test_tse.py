"""TSE and TSE_LIMIT interpolation (interp_s2u_r1, src/lp_tracking_m.f90:526-654): a Taylor
series about the tracked node with grad_sr1's central differences (src/gradient_m.f90:11-66),
TSE_LIMIT clamped to the 27 surrounding values.  The reference uses them for non-rectilinear
grids and accepts them as an INTERPOLATOR on any grid; here they run on rectilinear grids.

CPU: the oracle's restatement runs, differs from LINEAR and stays near it.  GPU: the library
against the oracle with the LINEAR parity bounds (flow map 1e-12 L, FTLE 1e-9 in FP64)."""
import numpy as np
import pytest

from libcfd2lcs_b200 import workloads as W
from tests import scenarios as SC

TSE, TSE_LIMIT = 5, 6


def _ftle(api, case, integrator, interp):
    api.reset()
    _, hs = SC.run(api, case, (SC.FTLE_BKWD, SC.FTLE_FWD), integrator, interp)
    return [api.ftle(h) for h in hs]


@pytest.mark.parametrize("case", ["dg", "abc_unsteady"])
def test_oracle_taylor_series_near_linear(oracle_dp, case):
    """Both interpolators are second-order accurate: on these grids their FTLE fields stay
    within a fifth of the field's range of LINEAR's, without being equal to it."""
    lin = _ftle(oracle_dp, case, 3, 1)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    for interp in (TSE, TSE_LIMIT):
        f = _ftle(oracle_dp, case, 3, interp)
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
        for a, b in zip(f, lin):
            assert np.all(np.isfinite(a))
            d = float(np.max(np.abs(a - b)))
            assert 1e-6 < d < 0.2 * float(np.ptp(b))
    oracle_dp.reset()


def test_oracle_limiter_changes_a_sheared_case(oracle_dp):
    """The limiter acts where the expansion overshoots its neighbourhood (mixed walls and
    periodic faces): TSE and TSE_LIMIT give different fields there."""
    a = _ftle(oracle_dp, "mixed_bc", 3, TSE)
    b = _ftle(oracle_dp, "mixed_bc", 3, TSE_LIMIT)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    assert max(float(np.max(np.abs(x - y))) for x, y in zip(a, b)) > 1e-6
    oracle_dp.reset()


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


@pytest.fixture(scope="module")
def gpu_sp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("sp")


CASES = [("dg", 2, TSE), ("dg", 3, TSE_LIMIT), ("abc_unsteady", 3, TSE), ("abc_unsteady", 2, TSE_LIMIT),
         ("mixed_bc", 3, TSE), ("mixed_bc", 3, TSE_LIMIT), ("channel", 2, TSE_LIMIT), ("turb", 2, TSE), ("dg", 4, TSE_LIMIT)]


@pytest.mark.gpu
@pytest.mark.parametrize("case,integrator,interp", CASES)
def test_taylor_series_matches_oracle(oracle_dp, gpu_dp, case, integrator, interp):
    from tests.test_gpu_parity import _compare
    try:
        _compare(oracle_dp, gpu_dp, case, integrator, interp, ftle_tol=1e-9)
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
@pytest.mark.parametrize("case,integrator,interp", [("abc_unsteady", 3, TSE_LIMIT), ("dg", 2, TSE)])
def test_taylor_series_single_precision(oracle_sp, gpu_sp, case, integrator, interp):
    from tests.test_gpu_parity import _compare
    try:
        _compare(oracle_sp, gpu_sp, case, integrator, interp, fm_tol_rel=2e-5, ftle_tol=3e-4)
    finally:
        gpu_sp.reset()


@pytest.mark.gpu
def test_taylor_series_mixed_precision(oracle_dp, gpu_dp):
    from tests.test_gpu_parity import _compare
    try:
        _compare(oracle_dp, gpu_dp, "dg", 2, TSE_LIMIT, fm_tol_rel=1e-6, ftle_tol=1e-5, mixed=True)
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
@pytest.mark.parametrize("case,res,integrator,interp", [("abc_unsteady", 1, 2, TSE_LIMIT), ("dg", 2, 3, TSE)])
def test_taylor_series_refined_grid(oracle_dp, gpu_dp, case, res, integrator, interp):
    """A refined lcs grid: the velocity expansion about the solver-grid node, the flow-map
    expansion about the lcs-grid node."""
    def run(api):
        g, vel, prm = SC.make_case(case)
        api.reset()
        api.init(g.n, g.x, g.y, g.z, g.flag)
        hs = [api.diagnostic_init(d, res, prm["T"], prm["h"], f"d{d}") for d in (SC.FTLE_BKWD, SC.FTLE_FWD)]
        api.set_option("INTEGRATOR", integrator)
        api.set_option("INTERPOLATOR", interp)
        for k in range(prm["steps"]):
            t = W.time_at(k, prm["dt"])
            api.update(*vel(t), t)
        return g, hs
    g, ho = run(oracle_dp)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        _, hg = run(gpu_dp)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        L = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
        for a, b in zip(ho, hg):
            assert gpu_dp.diag_size(b) == oracle_dp.diag_size(a)
            assert float(np.max(np.abs(oracle_dp.flowmap(a) - gpu_dp.flowmap(b)))) <= 1e-12 * L
            assert float(np.max(np.abs(oracle_dp.ftle(a) - gpu_dp.ftle(b)))) <= 1e-9
    finally:
        gpu_dp.reset()
