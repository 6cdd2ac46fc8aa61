"""Diagnostics on a refined or coarsened lcs grid (resolution /= 0 in cfd2lcs_diagnostic_init;
new_sgrid_from_sgrid, src/sgrid_m.f90:446-761; the flow map on the lcs grid, the velocity on the
solver grid, update_flowmap_sl, src/flowmap_m.f90:17-104): the oracle's grid rule (CPU) and the
library against the oracle (GPU)."""
import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _run(api, case, res, integrator, interp, directions=(SC.FTLE_BKWD, SC.FTLE_FWD), steps=None):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    hs = [api.diagnostic_init(d, res, prm["T"], prm["h"], f"d{d}") for d in directions]
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    for k in range(steps or prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return g, hs


def _expected_size(n, per, res):
    """Points per axis: res > 0 adds res per node, none past the last node of a non-periodic
    axis; res < 0 keeps every (|res|+1)-th node; singleton axes stay; |res| >= n resets to 0."""
    if any(m > 1 and abs(res) >= m for m in n):
        return tuple(n)
    out = []
    for m, p in zip(n, per):
        if m == 1:
            out.append(1)
        elif res > 0:
            out.append(m * (1 + res) - (0 if p else res))
        else:
            out.append(m // (abs(res) + 1))
    return tuple(out)


@pytest.mark.parametrize("case,res,per", [("abc_unsteady", 1, (1, 1, 1)), ("abc_unsteady", -1, (1, 1, 1)),
                                          ("dg", 2, (0, 0, 0)), ("mixed_bc", 1, (0, 1, 0)), ("abc_unsteady", 12, (1, 1, 1))])
def test_oracle_lcs_grid_size(oracle_dp, case, res, per):
    g, hs = _run(oracle_dp, case, res, 2, 1, steps=12)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    for h in hs:
        assert oracle_dp.diag_size(h) == _expected_size(g.n, per, res)
        assert np.all(np.isfinite(oracle_dp.ftle(h)))


def test_oracle_coarsened_flags_follow_the_reference(oracle_dp):
    """Coarsening the double gyre keeps interior (INTERNAL) nodes on its boundary faces, so the
    new grid's flags no longer agree with a wall: init_sgrid's periodicity check fails, as it
    does in the reference."""
    g, vel, prm = SC.make_case("dg")
    oracle_dp.reset()
    oracle_dp.init(g.n, g.x, g.y, g.z, g.flag)
    assert oracle_dp.diagnostic_init(SC.FTLE_BKWD, -1, prm["T"], prm["h"], "b") == -1
    assert "periodicity" in oracle_dp.error_msg()
    oracle_dp.reset()


CASES = [
    ("abc_unsteady", 1, 2, 1),
    ("abc_unsteady", -1, 3, 0),
    ("dg", 2, 2, 1),
    ("dg", 1, 4, 0),
    ("mixed_bc", 1, 3, 1),
    ("abc_unsteady", 1, 3, 3),
    ("dg", 2, 2, 3),
    ("mixed_bc", 1, 2, 2),
]
FTLE_TOL = {0: 1e-9, 1: 1e-9, 2: 1e-8, 3: 1e-8}


@pytest.mark.gpu
@pytest.mark.parametrize("case,res,integrator,interp", CASES)
def test_resolution_matches_oracle(oracle_dp, gpu_dp, case, res, integrator, interp):
    g, ho = _run(oracle_dp, case, res, integrator, interp)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        _, hg = _run(gpu_dp, case, res, integrator, interp)
        err, msg = gpu_dp.error()
        assert err == 0, msg
        L = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
        for a, b in zip(ho, hg):
            assert gpu_dp.diag_size(b) == oracle_dp.diag_size(a)
            fo, fg = oracle_dp.flowmap(a), gpu_dp.flowmap(b)
            to, tg = oracle_dp.ftle(a), gpu_dp.ftle(b)
            assert np.all(np.isfinite(tg))
            assert float(np.max(np.abs(fo - fg))) <= 1e-12 * L
            assert float(np.max(np.abs(to - tg))) <= FTLE_TOL[interp]
        cg = gpu_dp.counters()
        for k in ("integrations_fwd", "integrations_bkwd", "ftle_frames"):
            assert cg[k] == oracle_dp.counter(k), k
    finally:
        gpu_dp.reset()


def _run_opts(api, case, res, integrator, interp, opts):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    hs = [api.diagnostic_init(d, res, prm["T"], prm["h"], f"d{d}") for d in (SC.FTLE_BKWD, SC.FTLE_FWD)]
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    for k, v in opts.items():
        api.set_option(k, v)
    for k in range(prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return g, hs


@pytest.mark.gpu
@pytest.mark.parametrize("case,res,integrator,interp", [("abc_unsteady", 1, 2, 1), ("mixed_bc", 1, 3, 3), ("dg", 2, 2, 1)])
def test_resolution_invariants(oracle_dp, gpu_dp, case, res, integrator, interp):
    """compute_invariants on a refined lcs grid: lp%ugrid is the snapshot interpolated at the lcs
    nodes (reconstruct_flowmap); flags as in the solver-grid invariants test (lambda-2 ties
    excepted), H within 1e-9 relative."""
    _, ho = _run_opts(oracle_dp, case, res, integrator, interp, {"VELOCITY_INVARIANTS": 1})
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        _, hg = _run_opts(gpu_dp, case, res, integrator, interp, {"VELOCITY_INVARIANTS": 1})
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        for a, b in zip(ho, hg):
            io, ig = oracle_dp.invariants(a), gpu_dp.invariants(b)
            assert io.shape == ig.shape and io.shape[1:] == oracle_dp.diag_size(a)
            npts = io[0].size
            for q in (0, 1, 2):
                assert int(np.sum(io[q] != ig[q])) <= max(2, npts // 500), q
            off = io[4] != ig[4]
            assert np.all(np.abs(oracle_dp.l2margin(a)[off]) <= 1e-12)
            fin = np.isfinite(io[3]) & np.isfinite(ig[3])
            assert np.array_equal(np.isfinite(io[3]), np.isfinite(ig[3]))
            assert np.all(np.abs(io[3][fin] - ig[3][fin]) <= 1e-9 * np.maximum(1.0, np.abs(io[3][fin])))
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
def test_resolution_output_files(oracle_dp, gpu_dp, tmp_path, monkeypatch):
    """write_lcs on a refined lcs grid: the same files as the oracle's (names, headers with the
    lcs grid's sizes, grid and flag blocks identical text, the rest to the printed digits).
    CUBIC: with LINEAR interpolation the refined lp%ugrid of this flow is piecewise linear and
    many invariants are exactly zero, so their sign flags are set by last-bit rounding (in the
    reference too) and do not make a parity check."""
    import os

    from tests.test_writer import _compare_files
    opts = {"WRITE_LCS": 1, "WRITE_BCFLAG": 1, "VELOCITY_INVARIANTS": 1}
    odir = tmp_path / "o"
    odir.mkdir()
    oracle_dp.set_output_dir(str(odir))
    try:
        _run_opts(oracle_dp, "mixed_bc", 1, 3, 3, opts)
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
    finally:
        oracle_dp.set_output_dir("")
    gdir = tmp_path / "g"
    gdir.mkdir()
    monkeypatch.chdir(gdir)
    try:
        _run_opts(gpu_dp, "mixed_bc", 1, 3, 3, opts)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
    finally:
        gpu_dp.reset()
    names = sorted(os.listdir(odir))
    assert names and names == sorted(os.listdir(gdir / "cfd2lcs_output"))
    for nm in names:
        # lambda-2 (block 14) ties are common on this flow (the reference zeroes A(3,3)); its
        # parity is checked against the oracle's tie margin in test_resolution_invariants
        _compare_files(odir / nm, gdir / "cfd2lcs_output" / nm, rtol=2e-6, bitwise_blocks={0, 1, 2, 9}, flag_blocks={10, 11, 12},
                       skip_blocks={14})


@pytest.fixture(scope="module")
def gpu_sp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("sp")


@pytest.mark.gpu
@pytest.mark.parametrize("case,res,integrator,interp,aux", [("abc_unsteady", 1, 2, 1, 0), ("dg", 2, 3, 3, 0),
                                                            ("abc_unsteady", 0, 2, 1, 1)])
def test_single_precision_refined_and_aux(oracle_sp, gpu_sp, case, res, integrator, interp, aux):
    """The sp library (lcsdata_t = float) against the FP32 oracle on refined grids and with
    AUX_GRID: flow map within 2e-5 L; FTLE within 3e-4 (LINEAR), the single-precision parity
    bound, and within 1e-3 for the cubic case, whose 17,860-point refined grid carries FP32
    rounding of the B-spline fits through the FTLE's eigenvalue (measured 5.2e-4 there)."""
    def run(api):
        g, vel, prm = SC.make_case(case)
        api.reset()
        api.init(g.n, g.x, g.y, g.z, g.flag)
        api.set_option("AUX_GRID", aux)
        hs = [api.diagnostic_init(d, res, prm["T"], prm["h"], f"d{d}") for d in (SC.FTLE_BKWD, SC.FTLE_FWD)]
        api.set_option("INTEGRATOR", integrator)
        api.set_option("INTERPOLATOR", interp)
        for k in range(prm["steps"]):
            t = W.time_at(k, prm["dt"])
            api.update(*vel(t), t)
        return g, hs
    g, ho = run(oracle_sp)
    assert oracle_sp.error() == 0, oracle_sp.error_msg()
    try:
        _, hg = run(gpu_sp)
        err, msg = gpu_sp.error()
        assert err == 0, msg
        L = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)))
        for a, b in zip(ho, hg):
            assert float(np.max(np.abs(oracle_sp.flowmap(a) - gpu_sp.flowmap(b)))) <= 2e-5 * L
            assert float(np.max(np.abs(oracle_sp.ftle(a) - gpu_sp.ftle(b)))) <= (3e-4 if interp < 2 else 1e-3)
    finally:
        gpu_sp.reset()
