"""Host-side grid set-up of the library (tensor-product restatement of init_sgrid and
compute_delta_xyz) against the oracle's literal restatement: padded coordinates (fake,
periodic and extruded ghosts, including the z shift read at (i,k,k)), flags, boundary
normals and inverse half spans.  No GPU needed."""
import numpy as np
import pytest

import libcfd2lcs_b200 as L
from tests import workloads as W


def _mk(xl, yl, zl, fn=None):
    X, Y, Z = np.meshgrid(xl, yl, zl, indexing="ij")
    F = np.zeros(X.shape, dtype=np.int32)
    if fn:
        fn(F)
    return (len(xl), len(yl), len(zl)), np.asfortranarray(X), np.asfortranarray(Y), np.asfortranarray(Z), np.asfortranarray(F)


def _cases():
    rng = np.random.default_rng(1)
    c = {}
    g = W.double_gyre_grid(16, 8)
    c["double_gyre"] = (g.n, g.x, g.y, g.z, g.flag)
    g = W.abc_grid(8)
    c["abc_periodic"] = (g.n, g.x, g.y, g.z, g.flag)

    def chan(F):
        F[:, 0, :] = W.LCS_WALL
        F[:, -1, :] = W.LCS_WALL

    c["channel_z_periodic_y_walls"] = _mk(np.arange(6) * 0.3, np.cumsum(rng.uniform(0.5, 1.5, 7)), np.arange(5) * 0.25, chan)

    def slipy(F):
        F[:, 0, :] = W.LCS_SLIP
        F[:, -1, :] = W.LCS_SLIP

    c["nonuniform_periodic_x"] = _mk(np.cumsum(rng.uniform(0.5, 1.5, 6)), np.arange(5) * 0.2, np.arange(4) * 0.3, slipy)

    def mixed(F):
        F[0] = W.LCS_INFLOW
        F[-1] = W.LCS_OUTFLOW
        F[:, 0] = W.LCS_WALL
        F[:, -1] = W.LCS_SLIP
        F[2, 2, 1] = W.LCS_MASK
        F[3, 2, 1] = W.LCS_MASK

    c["mixed_flags"] = _mk(np.arange(7) * 0.1, np.arange(6) * 0.15, np.arange(4) * 0.2, mixed)
    c["x_singleton"] = _mk(np.array([0.5]), np.arange(6) * 0.2, np.arange(7) * 0.1)

    def ysing(F):
        F[0] = W.LCS_SLIP
        F[-1] = W.LCS_SLIP
        F[3, 0, 3] = W.LCS_MASK

    c["y_singleton_z_periodic"] = _mk(np.arange(6) * 0.2, np.array([0.5]), np.arange(7) * 0.1, ysing)
    return c


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_grid_tables_match_oracle(oracle_dp, name):
    n, x, y, z, f = CASES[name]
    oracle_dp.reset()
    oracle_dp.init(n, x, y, z, f)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    go = oracle_dp.grid_state()
    gp = L.Cfd2lcs("dp").grid_tables(n, x, y, z, f)
    assert np.array_equal(go["periodic"], gp["periodic"])
    assert np.array_equal(go["xyz"], gp["xyz"])
    assert np.array_equal(go["flag"], gp["flag"])
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    assert np.array_equal(go["inv_delta"][inner], gp["inv_delta"][inner])
    sel = np.isin(go["flag"], [W.LCS_WALL, W.LCS_SLIP, W.LCS_MASK])
    sel[0], sel[-1], sel[:, 0], sel[:, -1], sel[:, :, 0], sel[:, :, -1] = False, False, False, False, False, False
    assert np.max(np.abs(go["bcnorm"][:, sel] - gp["bcnorm"][:, sel]), initial=0.0) <= 1e-15


def test_grid_classes_and_bad_periodicity():
    api = L.Cfd2lcs("dp")
    n, x, y, z, f = CASES["abc_periodic"]
    x2 = x.copy()
    x2[3, 2, 1] += 1e-3  # 1.6e-4 of the domain: non-rectilinear, the full-array (least-squares) form
    assert api.grid_lsq_weights(n, x2, y, z, f)[0]
    x3 = x.copy()
    x3[3, 2, 1] += 1e-6  # within check_rectilinear's 1e-4 but not a tensor product: refused
    with pytest.raises(ValueError, match="tensor product"):
        api.grid_tables(n, x3, y, z, f)
    f2 = f.copy()
    f2[0, :, :] = W.LCS_WALL  # one x face walled, the other internal
    with pytest.raises(ValueError, match="eriodicity"):
        api.grid_tables(n, x, y, z, f2)
