"""TSE and TSE_LIMIT interpolation (interp_s2u_r1, src/lp_tracking_m.f90:526-654): a Taylor
series about the tracked node with grad_sr1's central differences (src/gradient_m.f90:11-66),
TSE_LIMIT clamped to the 27 surrounding values.  The reference uses them for non-rectilinear
grids and accepts them as an INTERPOLATOR on any grid; here they run on rectilinear grids.

CPU: known answers for the oracle's restatement (exact for affine fields about interior nodes,
the node value at a ghost node, no term along a singleton axis, the limiter as a clamp to the
27-value neighbourhood), and whole runs that differ from LINEAR but stay near it.  GPU: the
library against the oracle with the LINEAR parity bounds (flow map 1e-12 L, FTLE 1e-9 in FP64)."""
import numpy as np
import pytest

from tests import workloads as W
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


def _grid_case(oracle, case):
    g, _, _ = SC.make_case(case)
    oracle.reset()
    oracle.init(g.n, g.x, g.y, g.z, g.flag)
    assert oracle.error() == 0, oracle.error_msg()
    return g, oracle.grid_state()["xyz"]


def _interior_points(g, xyz, rng, m):
    """m random points within half a cell of random interior nodes, with those nodes."""
    no = np.stack([rng.integers(1, n + 1, m) for n in g.n])
    pts = np.empty((3, m))
    for a in range(3):
        base = xyz[a][no[0], no[1], no[2]]
        if g.n[a] == 1:
            pts[a] = base
            continue
        e = np.zeros((3, m), dtype=int)
        e[a] = 1
        up = xyz[a][no[0] + e[0], no[1] + e[1], no[2] + e[2]]
        dn = xyz[a][no[0] - e[0], no[1] - e[1], no[2] - e[2]]
        s = rng.uniform(-0.5, 0.5, m)
        pts[a] = base + np.where(s > 0, s * (up - base), -s * (dn - base))
    return pts, no


@pytest.mark.parametrize("case", ["channel", "mixed_bc"])
def test_oracle_taylor_series_exact_for_affine_fields(oracle_dp, case):
    """Central differences are exact for an affine field on any rectilinear spacing, so the
    expansion about an interior node reproduces the field at the point (TSE), and no limiter
    acts within half a cell of the node (TSE_LIMIT)."""
    g, xyz = _grid_case(oracle_dp, case)
    rng = np.random.default_rng(11)
    A, b = rng.normal(size=(3, 3)), rng.normal(size=3)
    f3 = np.einsum("ca,aijk->cijk", A, xyz) + b[:, None, None, None]
    pts, no = _interior_points(g, xyz, rng, 400)
    exact = A @ pts + b[:, None]
    for m in (TSE, TSE_LIMIT):
        out = oracle_dp.interp_points(m, f3, pts, no)
        np.testing.assert_allclose(out, exact, rtol=0, atol=1e-12 * float(np.max(np.abs(exact))))
    oracle_dp.reset()


def test_oracle_taylor_series_ghost_node_and_singleton_axis(oracle_dp):
    """The gradient is zero at a ghost node (grad_sr1 fills interior nodes only) and along a
    singleton axis (the double gyre's z): the expansion returns the node value there, and only
    the in-plane terms elsewhere."""
    g, xyz = _grid_case(oracle_dp, "dg")
    rng = np.random.default_rng(12)
    A, b = rng.normal(size=(3, 3)), rng.normal(size=3)
    f3 = np.einsum("ca,aijk->cijk", A, xyz) + b[:, None, None, None]
    ghost = np.array([[0, g.n[0] + 1, 3], [2, 5, 0], [1, 1, 1]])
    pts = np.stack([xyz[a][ghost[0], ghost[1], ghost[2]] for a in range(3)]) + 0.01
    node = f3[:, ghost[0], ghost[1], ghost[2]]
    for m in (TSE, TSE_LIMIT):
        np.testing.assert_array_equal(oracle_dp.interp_points(m, f3, pts, ghost), node)
    pts, no = _interior_points(g, xyz, rng, 50)
    pts[2] += 0.3  # off the data plane: no z term
    node = f3[:, no[0], no[1], no[2]]
    want = node + A[:, :2] @ (pts[:2] - np.stack([xyz[a][no[0], no[1], no[2]] for a in range(2)]))
    np.testing.assert_allclose(oracle_dp.interp_points(TSE, f3, pts, no), want, rtol=0, atol=1e-12)
    oracle_dp.reset()


def test_oracle_limiter_clamps_to_the_neighbourhood(oracle_dp):
    """TSE_LIMIT is TSE clamped to the range of the 27 values around the node (clipped to the
    padded array)."""
    g, xyz = _grid_case(oracle_dp, "channel")
    rng = np.random.default_rng(13)
    f3 = rng.normal(size=(3,) + xyz.shape[1:])
    pts, no = _interior_points(g, xyz, rng, 300)
    t = oracle_dp.interp_points(TSE, f3, pts, no)
    lim = oracle_dp.interp_points(TSE_LIMIT, f3, pts, no)
    n = np.array(g.n)
    for q in range(pts.shape[1]):
        lo = np.maximum(no[:, q] - 1, 0)
        hi = np.minimum(no[:, q] + 1, n + 1)
        win = f3[:, lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1].reshape(3, -1)
        np.testing.assert_array_equal(lim[:, q], np.minimum(np.maximum(t[:, q], win.min(1)), win.max(1)))
    assert np.any(lim != t)
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
