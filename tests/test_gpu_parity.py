"""Parity of the CUDA path (libcfd2lcs_b200, called through its C ABI) with the oracle
(the CPU restatement of the reference) on seeded synthetic flows at small sizes.

Tolerances:
  plain FP64 (dp library) vs the FP64 oracle: composed flow map max-abs <= 1e-12 * L (L the
    domain length), FTLE max-abs <= 1e-9 for LINEAR / NEAREST and <= 1e-8 for the B-splines;
  plain FP32 (sp library) vs the FP32 oracle: flow map <= 2e-5 * L, FTLE <= 3e-4 (both round
    every operation in FP32, the device with FMA contraction, the oracle without);
  mixed precision (dp library, MIXED_PRECISION = 1: FP32 velocity data) vs the FP64 oracle:
    flow map <= 1e-6 * L, FTLE <= 1e-5.
"""
import numpy as np
import pytest

from tests import scenarios as SC

pytestmark = pytest.mark.gpu

FM_TOL_REL = 1e-12
FTLE_TOL = {0: 1e-9, 1: 1e-9, 2: 1e-8, 3: 1e-8}


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


@pytest.fixture(scope="module")
def gpu_sp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("sp")


def _compare(oracle, gpu, case, integrator, interpolator, directions=(SC.FTLE_BKWD, SC.FTLE_FWD), n=None, steps=None,
             fm_tol_rel=FM_TOL_REL, ftle_tol=None, mixed=False):
    oracle.reset()
    g, ho = SC.run(oracle, case, directions, integrator, interpolator, n=n, steps=steps)
    assert oracle.error() == 0, oracle.error_msg()
    gpu.reset()
    if mixed:
        gpu.set_option("MIXED_PRECISION", 1)
    _, hg = SC.run(gpu, case, directions, integrator, interpolator, n=n, steps=steps)
    err, msg = gpu.error()
    assert err == 0, msg
    L = max(float(np.ptp(g.x)), float(np.ptp(g.y)), float(np.ptp(g.z)), 1e-30)
    out = {}
    for d, a, b in zip(directions, ho, hg):
        fo, fg = oracle.flowmap(a), gpu.flowmap(b)
        to, tg = oracle.ftle(a), gpu.ftle(b)
        dfm = float(np.max(np.abs(fo - fg)))
        dft = float(np.max(np.abs(to - tg)))
        out[d] = (dfm, dft)
        assert np.all(np.isfinite(tg))
        tol = FTLE_TOL[interpolator] if ftle_tol is None else ftle_tol
        assert dfm <= fm_tol_rel * L, f"flow map max-abs {dfm:.3e} (dir {d}) > {fm_tol_rel * L:.3e}"
        assert dft <= tol, f"FTLE max-abs {dft:.3e} (dir {d}) > {tol:.1e}"
    cg, co = gpu.counters(), {k: oracle.counter(k) for k in ("integrations_fwd", "integrations_bkwd", "ftle_frames")}
    for k in co:
        assert cg[k] == co[k], (k, cg[k], co[k])
    return out


@pytest.mark.parametrize("integrator", [2, 3])
def test_double_gyre_linear(oracle_dp, gpu_dp, integrator):
    _compare(oracle_dp, gpu_dp, "dg", integrator, 1)


@pytest.mark.parametrize("integrator", [0, 1, 4])
def test_double_gyre_other_integrators(oracle_dp, gpu_dp, integrator):
    _compare(oracle_dp, gpu_dp, "dg", integrator, 1, n=32, steps=20)


def test_double_gyre_nearest(oracle_dp, gpu_dp):
    _compare(oracle_dp, gpu_dp, "dg", 2, 0, n=32, steps=20)


@pytest.mark.parametrize("integrator", [2, 3])
def test_abc_linear(oracle_dp, gpu_dp, integrator):
    _compare(oracle_dp, gpu_dp, "abc", integrator, 1)


@pytest.mark.parametrize("interp", [2, 3])
def test_abc_spline(oracle_dp, gpu_dp, interp):
    _compare(oracle_dp, gpu_dp, "abc", 3, interp, n=12, steps=12)


def test_abc_unsteady_rk4_cubic(oracle_dp, gpu_dp):
    _compare(oracle_dp, gpu_dp, "abc_unsteady", 4, 3, n=10, steps=10)


def test_double_gyre_cubic(oracle_dp, gpu_dp):
    _compare(oracle_dp, gpu_dp, "dg", 3, 3, n=32, steps=20)


def test_channel_walls_zquirk(oracle_dp, gpu_dp):
    _compare(oracle_dp, gpu_dp, "channel", 2, 1)


def test_channel_cubic_is_rejected_like_the_oracle(oracle_dp, gpu_dp):
    """Periodic z with walled y: the reference's unshifted periodic z ghosts make the spline
    abscissae non-increasing (db3ink input check fails and the coefficients are undefined);
    the oracle and the library both refuse the spline interpolators there."""
    oracle_dp.reset()
    SC.run(oracle_dp, "channel", (SC.FTLE_BKWD,), 2, 3, steps=3)
    assert oracle_dp.error() == 1
    gpu_dp.reset()
    SC.run(gpu_dp, "channel", (SC.FTLE_BKWD,), 2, 3, steps=3)
    err, msg = gpu_dp.error()
    assert err == 1 and "bspline" in msg
    gpu_dp.reset()


@pytest.mark.parametrize("interp", [1, 3])
def test_mixed_boundary_conditions(oracle_dp, gpu_dp, interp):
    _compare(oracle_dp, gpu_dp, "mixed_bc", 3, interp)


@pytest.mark.parametrize("integrator,interp", [(2, 1), (3, 3)])
def test_turbulence(oracle_dp, gpu_dp, integrator, interp):
    _compare(oracle_dp, gpu_dp, "turb", integrator, interp)


@pytest.mark.parametrize("case,integrator,interp", [("dg", 2, 1), ("abc", 3, 3), ("turb", 2, 1), ("mixed_bc", 3, 1)])
def test_single_precision_build(oracle_sp, gpu_sp, case, integrator, interp):
    """The sp library (lcsdata_t = float) against the FP32 oracle."""
    _compare(oracle_sp, gpu_sp, case, integrator, interp, fm_tol_rel=2e-5, ftle_tol=3e-4)


@pytest.mark.parametrize("case,integrator,interp", [("dg", 2, 1), ("abc", 3, 3), ("turb", 3, 3), ("abc_unsteady", 4, 3)])
def test_mixed_precision_form(oracle_dp, gpu_dp, case, integrator, interp):
    """MIXED_PRECISION = 1 (FP32 velocity levels, coefficients and tap contractions; FP64
    positions, flow maps and FTLE) against the FP64 oracle."""
    try:
        _compare(oracle_dp, gpu_dp, case, integrator, interp, fm_tol_rel=1e-6, ftle_tol=1e-5, mixed=True)
    finally:
        gpu_dp.reset()


def _run_with_invariants(api, case, directions, integrator, interpolator):
    from tests import workloads as W
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    hs = [api.diagnostic_init(d, 0, prm["T"], prm["h"], f"d{d}") for d in directions]
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interpolator)
    api.set_option("VELOCITY_INVARIANTS", 1)
    for k in range(prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return hs


@pytest.mark.parametrize("case,integrator,interp", [("abc_unsteady", 2, 1), ("mixed_bc", 3, 1), ("dg", 2, 3), ("turb", 3, 3)])
def test_velocity_invariants(oracle_dp, gpu_dp, case, integrator, interp):
    """compute_invariants (VELOCITY_INVARIANTS): Q, D, C and lambda-2 flags equal the oracle's
    (allowing a point or two where an invariant sits at zero within rounding), H within 1e-9
    relative where finite."""
    dirs = (SC.FTLE_BKWD, SC.FTLE_FWD)
    ho = _run_with_invariants(oracle_dp, case, dirs, integrator, interp)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    try:
        hg = _run_with_invariants(gpu_dp, case, dirs, integrator, interp)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        for a, b in zip(ho, hg):
            io, ig = oracle_dp.invariants(a), gpu_dp.invariants(b)
            npts = io[0].size
            for q in (0, 1, 2):
                mism = int(np.sum(io[q] != ig[q]))
                assert mism <= max(2, npts // 500), (q, mism)
            # lambda-2: the reference zeroes A(3,3), so exact-arithmetic ties (middle eigenvalue
            # 0) are common and their sign is rounding noise; disagreement only at such ties
            off = io[4] != ig[4]
            assert np.all(np.abs(oracle_dp.l2margin(a)[off]) <= 1e-12), np.abs(oracle_dp.l2margin(a)[off]).max()
            fin = np.isfinite(io[3]) & np.isfinite(ig[3])
            assert np.array_equal(np.isfinite(io[3]), np.isfinite(ig[3]))
            assert np.all(np.abs(io[3][fin] - ig[3][fin]) <= 1e-9 * np.maximum(1.0, np.abs(io[3][fin])))
    finally:
        gpu_dp.reset()


@pytest.mark.parametrize("case,integrator,directions", [("abc_unsteady", 2, (SC.FTLE_BKWD, SC.FTLE_FWD)), ("dg", 3, (SC.FTLE_BKWD,)),
                                                        ("mixed_bc", 4, (SC.FTLE_BKWD, SC.FTLE_FWD)),
                                                        # forward set first: its blends must not leak into the backward set
                                                        ("abc_unsteady", 3, (SC.FTLE_FWD, SC.FTLE_BKWD))])
def test_linear_stage_blends(oracle_dp, gpu_dp, case, integrator, directions, monkeypatch):
    """LINEAR with the stage blends written once per subcycle (the large-grid path, forced on
    small grids through CFD2LCS_B200_LINEAR_BLEND_MIN): the same parity bounds."""
    monkeypatch.setenv("CFD2LCS_B200_LINEAR_BLEND_MIN", "0")
    _compare(oracle_dp, gpu_dp, case, integrator, 1, directions=directions)
