"""AUX_GRID (create_aux_grid, src/lcs_m.f90:225-435; the auxiliary-grid Cauchy-Green gradient,
src/lcs_m.f90:95-127): six auxiliary particle sets per diagnostic, shifted by a fifth of the
mean neighbour distance along each axis.  The oracle's restatement (CPU) and the library
against it (GPU)."""
import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _run(api, case, integrator, interp, aux=1, res=0, directions=(SC.FTLE_BKWD, SC.FTLE_FWD), steps=None, aux_after=False):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    if not aux_after:
        api.set_option("AUX_GRID", aux)
    hs = [api.diagnostic_init(d, res, prm["T"], prm["h"], f"d{d}") for d in directions]
    if aux_after:
        api.set_option("AUX_GRID", aux)
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    for k in range(steps or prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return g, hs


def test_oracle_aux_sets_are_advected(oracle_dp):
    """Seven particle sets per diagnostic (the set and its six auxiliary ones), all counted as
    set_dt counts every set; the AUX FTLE is finite and close to the central-difference one."""
    _run(oracle_dp, "abc_unsteady", 2, 1, aux=0, directions=(SC.FTLE_BKWD,))
    plain = oracle_dp.counter("integrations_bkwd")
    f0 = oracle_dp.ftle(1)
    _run(oracle_dp, "abc_unsteady", 2, 1, aux=1, directions=(SC.FTLE_BKWD,))
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    assert oracle_dp.counter("integrations_bkwd") == 7 * plain
    f1 = oracle_dp.ftle(1)
    assert np.all(np.isfinite(f1))
    assert float(np.mean(np.abs(f1 - f0))) < 0.1 * float(np.mean(np.abs(f0)))


def test_oracle_aux_set_after_init_is_an_error(oracle_dp):
    _run(oracle_dp, "abc_unsteady", 2, 1, aux_after=True, directions=(SC.FTLE_BKWD,))
    assert oracle_dp.error() != 0 and "AUX_GRID" in oracle_dp.error_msg()
    oracle_dp.reset()


CASES = [
    ("abc_unsteady", 2, 1, 0),
    ("abc", 3, 3, 0),
    ("turb", 3, 1, 0),
    ("abc_unsteady", 2, 1, 1),
    ("abc_unsteady", 3, 5, 0),
]
FTLE_TOL = {0: 1e-9, 1: 1e-9, 2: 1e-8, 3: 1e-8, 5: 1e-9, 6: 1e-9}


@pytest.mark.gpu
@pytest.mark.parametrize("case,integrator,interp,res", CASES)
def test_aux_grid_matches_oracle(oracle_dp, gpu_dp, case, integrator, interp, res):
    g, ho = _run(oracle_dp, case, integrator, interp, res=res)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        _, hg = _run(gpu_dp, case, integrator, interp, res=res)
        err, msg = gpu_dp.error()
        assert err == 0, msg
        assert hg == ho
        for a, b in zip(ho, hg):
            to, tg = oracle_dp.ftle(a), gpu_dp.ftle(b)
            assert np.all(np.isfinite(tg))
            assert float(np.max(np.abs(to - tg))) <= FTLE_TOL[interp]
        cg = gpu_dp.counters()
        for k in ("integrations_fwd", "integrations_bkwd", "ftle_frames"):
            assert cg[k] == oracle_dp.counter(k), k
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
def test_aux_grid_errors(gpu_dp):
    """Set after the diagnostic exists: the frame latches an error.  Non-uniform spacing (the
    double gyre's boundary nodes): the auxiliary grids are not tensor products, rejected at
    cfd2lcs_diagnostic_init."""
    _run(gpu_dp, "abc_unsteady", 2, 1, aux_after=True, directions=(SC.FTLE_BKWD,))
    err, msg = gpu_dp.error()
    assert err != 0 and "AUX_GRID" in msg
    g, vel, prm = SC.make_case("dg")
    gpu_dp.reset()
    gpu_dp.init(g.n, g.x, g.y, g.z, g.flag)
    gpu_dp.set_option("AUX_GRID", 1)
    assert gpu_dp.diagnostic_init(SC.FTLE_BKWD, 0, prm["T"], prm["h"], "b") == -1
    err, msg = gpu_dp.error()
    assert err != 0 and "tensor product" in msg
    gpu_dp.reset()
