"""Parity of the CUDA path with the oracle on non-rectilinear grids: the reference's
least-squares path (TSE_LIMIT in place of every interpolator but TSE, src/lp_tracking_m.f90:
320-327; grad_sr1_ls for the Taylor series, the FTLE and the invariants, src/gradient_m.f90:
241-295; the node search, boundary conditions and 2-D plane projection on full coordinate
arrays; exchange_lp_alltoall's node guess of src/comms_m.f90:1662-1673).

Tolerances as the rectilinear Taylor-series cases: plain FP64 vs the FP64 oracle, flow map
max-abs <= 1e-12 * L and FTLE max-abs <= 1e-9; FP32 vs the FP32 oracle 2e-5 * L / 3e-4;
mixed precision vs the FP64 oracle 1e-6 * L / 1e-5."""
import numpy as np
import pytest

from tests import scenarios as SC
from tests.test_gpu_parity import _compare

pytestmark = pytest.mark.gpu

TSE, TSE_LIMIT = 5, 6


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


@pytest.fixture(scope="module")
def gpu_sp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("sp")


@pytest.mark.parametrize("case", ["curv_box", "curv_periodic", "curv_dg"])
@pytest.mark.parametrize("integrator", [2, 3])
@pytest.mark.parametrize("interp", [1, TSE])  # LINEAR runs as TSE_LIMIT on these grids
def test_curvilinear_matches_oracle(oracle_dp, gpu_dp, case, integrator, interp):
    _compare(oracle_dp, gpu_dp, case, integrator, interp, ftle_tol=1e-9)


@pytest.mark.parametrize("integrator", [0, 1, 4])
def test_curvilinear_other_integrators(oracle_dp, gpu_dp, integrator):
    _compare(oracle_dp, gpu_dp, "curv_box", integrator, TSE_LIMIT, ftle_tol=1e-9, steps=10)


def test_curvilinear_cubic_request_runs_tse_limit(gpu_dp):
    # CUBIC on a non-rectilinear grid gives bitwise what TSE_LIMIT gives
    out = []
    for interp in (3, TSE_LIMIT):
        gpu_dp.reset()
        _, h = SC.run(gpu_dp, "curv_periodic", (SC.FTLE_BKWD,), 2, interp, steps=10)
        err, msg = gpu_dp.error()
        assert err == 0, msg
        out.append(gpu_dp.ftle(h[0]))
    assert np.array_equal(out[0], out[1])


def test_curvilinear_single_precision(oracle_sp, gpu_sp):
    _compare(oracle_sp, gpu_sp, "curv_box", 2, TSE_LIMIT, fm_tol_rel=2e-5, ftle_tol=3e-4)


def test_curvilinear_mixed_precision(oracle_dp, gpu_dp):
    _compare(oracle_dp, gpu_dp, "curv_dg", 2, TSE_LIMIT, fm_tol_rel=1e-6, ftle_tol=1e-5, mixed=True)


def test_curvilinear_sorted_composition(oracle_dp, gpu_dp):
    # the one-step-per-sub-map composition with particle re-sorting (the large-grid path),
    # forced on a small grid; the environment is read at cfd2lcs_init
    import os
    os.environ["CFD2LCS_B200_COMPOSE_SORT_MIN"] = "0"
    try:
        _compare(oracle_dp, gpu_dp, "curv_periodic", 2, TSE_LIMIT, n=20, steps=10, ftle_tol=1e-9)
    finally:
        os.environ.pop("CFD2LCS_B200_COMPOSE_SORT_MIN", None)


def test_curvilinear_invariants(oracle_dp, gpu_dp):
    """compute_invariants with grad_sr1_ls: the same checks as the rectilinear invariants test."""
    from tests.test_gpu_parity import _run_with_invariants
    dirs = (SC.FTLE_BKWD,)
    ho = _run_with_invariants(oracle_dp, "curv_box", dirs, 2, TSE_LIMIT)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        hg = _run_with_invariants(gpu_dp, "curv_box", dirs, 2, TSE_LIMIT)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        io, ig = oracle_dp.invariants(ho[0]), gpu_dp.invariants(hg[0])
        npts = io[0].size
        for q in (0, 1, 2):
            assert int(np.sum(io[q] != ig[q])) <= max(2, npts // 500), q
        off = io[4] != ig[4]
        assert np.all(np.abs(oracle_dp.l2margin(ho[0])[off]) <= 1e-12)
        fin = np.isfinite(io[3]) & np.isfinite(ig[3])
        assert np.array_equal(np.isfinite(io[3]), np.isfinite(ig[3]))
        assert np.all(np.abs(io[3][fin] - ig[3][fin]) <= 1e-9 * np.maximum(1.0, np.abs(io[3][fin])))
    finally:
        gpu_dp.reset()


@pytest.mark.parametrize("opt", ["resolution", "aux"])
def test_curvilinear_unsupported_options_latch(gpu_dp, opt):
    g = SC.curvilinear_grid("curv_box")
    gpu_dp.reset()
    gpu_dp.init(g.n, g.x, g.y, g.z, g.flag)
    if opt == "aux":
        gpu_dp.set_option("AUX_GRID", 1)
        gpu_dp.diagnostic_init(SC.FTLE_BKWD, 0, 0.6, 0.2, "a")
    else:
        gpu_dp.diagnostic_init(SC.FTLE_BKWD, 1, 0.6, 0.2, "r")
    err, msg = gpu_dp.error()
    assert err != 0 and "non-rectilinear" in msg
    gpu_dp.reset()
