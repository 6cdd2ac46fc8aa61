"""Non-rectilinear (curvilinear) grids on the host: the library's padded coordinates (the
reference's ghost construction on full arrays), inverse half spans, boundary normals and
face-neighbour least-squares weights (compute_lsgw, src/gradient_m.f90:114-217) against the
oracle's restatement, bit for bit; the grids that check_rectilinear (src/sgrid_m.f90:868-949)
classes as rectilinear without being exact tensor products are refused.  No GPU needed."""
import numpy as np
import pytest

import libcfd2lcs_b200 as L
from tests import workloads as W
from tests import scenarios as SC

CASES = ("curv_box", "curv_periodic", "curv_dg")


@pytest.mark.parametrize("case", CASES)
def test_curvilinear_tables_match_oracle(oracle_dp, case):
    g = SC.curvilinear_grid(case)
    oracle_dp.reset()
    oracle_dp.init(g.n, g.x, g.y, g.z, g.flag)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    go = oracle_dp.grid_state()
    rect, wo = oracle_dp.lsq_weights()
    lib = L.Cfd2lcs("dp")
    gp = lib.grid_tables(g.n, g.x, g.y, g.z, g.flag)
    curv, wp = lib.grid_lsq_weights(g.n, g.x, g.y, g.z, g.flag)
    assert not rect and curv
    assert np.array_equal(go["periodic"], gp["periodic"])
    assert np.array_equal(go["xyz"], gp["xyz"])
    assert np.array_equal(go["flag"], gp["flag"])
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    assert np.array_equal(go["inv_delta"][inner], gp["inv_delta"][inner])
    assert np.array_equal(wo, wp)
    # weights vanish on the ghost layer and reproduce the gradient of a linear field exactly
    # up to rounding at interior nodes
    assert not np.any(wp[:, :, 0]) and not np.any(wp[:, :, -1])
    sel = np.isin(go["flag"], [W.LCS_WALL, W.LCS_SLIP, W.LCS_MASK])
    sel[0], sel[-1], sel[:, 0], sel[:, -1], sel[:, :, 0], sel[:, :, -1] = False, False, False, False, False, False
    assert np.max(np.abs(go["bcnorm"][:, sel] - gp["bcnorm"][:, sel]), initial=0.0) <= 1e-15


def test_least_squares_weights_are_exact_for_affine_fields():
    g = SC.curvilinear_grid("curv_box")
    curv, w = L.Cfd2lcs("dp").grid_lsq_weights(g.n, g.x, g.y, g.z, g.flag)
    xyz = L.Cfd2lcs("dp").grid_tables(g.n, g.x, g.y, g.z, g.flag)["xyz"]
    coef = np.array([0.7, -1.3, 2.1])
    f = np.tensordot(coef, xyz, axes=1) + 0.4
    offs = [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    ni, nj, nk = g.n
    core = (slice(1, ni + 1), slice(1, nj + 1), slice(1, nk + 1))
    grad = np.zeros((3,) + f[core].shape)
    for nb, (a, b, c) in enumerate(offs):
        sh = f[1 + a:ni + 1 + a, 1 + b:nj + 1 + b, 1 + c:nk + 1 + c] - f[core]
        for comp in range(3):
            grad[comp] += sh * w[nb, comp][core]
    for comp in range(3):
        assert np.max(np.abs(grad[comp] - coef[comp])) < 1e-11


def test_nearly_rectilinear_grid_is_refused():
    # within check_rectilinear's 1e-4 tolerance but not an exact tensor product: the reference
    # runs its rectilinear path on the coordinate lines through node 1, which this library does
    # not reproduce; it refuses the grid with an error instead
    g = W.abc_grid(8)
    x = np.asfortranarray(g.x + 1e-7 * np.sin(g.y))
    with pytest.raises(ValueError, match="tolerance"):
        L.Cfd2lcs("dp").grid_tables(g.n, x, g.y, g.z, g.flag)


@pytest.mark.parametrize("case", CASES)
def test_oracle_runs_curvilinear_cases(oracle_dp, case):
    # TSE_LIMIT replaces LINEAR on these grids, TSE stays TSE (src/lp_tracking_m.f90:320-327)
    for interp in (1, 5):
        oracle_dp.reset()
        g, h = SC.run(oracle_dp, case, integrator=2, interpolator=interp, steps=8)
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
        for x in h:
            assert np.all(np.isfinite(oracle_dp.ftle(x)))
    # LINEAR and NEAREST give the same result: both become TSE_LIMIT
    res = []
    for interp in (0, 1):
        oracle_dp.reset()
        g, h = SC.run(oracle_dp, case, integrator=2, interpolator=interp, steps=8)
        res.append(oracle_dp.ftle(h[0]))
    assert np.array_equal(res[0], res[1])
