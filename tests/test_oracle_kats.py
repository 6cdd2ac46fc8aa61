"""Known-answer tests of the oracle (the CPU restatement of the reference path).

The reference has no golden vectors, so parity of the oracle itself is pinned by answers
that follow from the reference's algorithm exactly: translation, the discrete rigid
rotation (which also pins the displacement-gradient FTLE of src/lcs_m.f90:128-176),
polynomial reproduction of the not-a-knot B-spline, and the eigen-solve against LAPACK."""
import math

import numpy as np
import pytest

from tests import workloads as W
from tests import kats


def test_translation_periodic(oracle_dp):
    o = oracle_dp
    o.reset()
    g = W.abc_grid(12)
    o.init(g.n, g.x, g.y, g.z, g.flag)
    hb = o.diagnostic_init(1, 0, 1.0, 0.5, "b")
    hf = o.diagnostic_init(0, 0, 1.0, 0.5, "f")
    U = (0.3, -0.2, 0.1)
    for k in range(21):
        o.update(*(np.full(g.n, c, order="F") for c in U), k * 0.05)
    assert o.error() == 0
    fb, ff = o.flowmap(hb), o.flowmap(hf)
    for c in range(3):
        assert np.max(np.abs(fb[c] + U[c] * 1.0)) < 1e-12
        assert np.max(np.abs(ff[c] - U[c] * 1.0)) < 1e-12
    # uniform displacement: the gradient vanishes up to rounding, FTLE is very negative
    assert o.ftle(hb).max() < -20.0


@pytest.mark.parametrize("integrator", [2, 3, 4])
def test_rigid_rotation_displacement_gradient_ftle(oracle_dp, integrator):
    o = oracle_dp
    o.reset()
    g, (u, v, w), A = kats.rotation_case(64, omega=0.5)
    T, h, dt = 1.0, 0.5, 0.05
    o.init(g.n, g.x, g.y, g.z, g.flag)
    hb = o.diagnostic_init(1, 0, T, h, "b")
    o.set_option("INTEGRATOR", integrator)
    nsub_total = 0
    for k in range(21):
        o.update(u, v, w, k * dt)
        if k > 0:
            nsub_total += o.counter("nsub_bkwd")
    assert o.error() == 0
    # steps 1..20 cover t in (0, 1]; the frame at t=1 composes slots 1 (t=0.5) and 0 (t=1.0)
    nsub = o.counter("nsub_bkwd")
    expect = kats.expected_ftle_linear(A, -dt / nsub, nsub_total, integrator, T)
    f = o.ftle(hb)
    inner = f[24:40, 24:40, 0]  # away from the slip walls, whose ghosts are not linear
    assert np.max(np.abs(inner - expect)) < 1e-11, (inner.min(), inner.max(), expect)
    # the textbook FTLE (gradient of the map, not of the displacement) would be ~0 here
    assert expect < -0.5


@pytest.mark.parametrize("order", [3, 4])
def test_bspline_reproduces_polynomials(oracle_dp, order):
    rng = np.random.default_rng(3)
    xg = np.sort(rng.uniform(0, 1, 9)); xg[0], xg[-1] = 0.0, 1.0
    yg = np.linspace(-1, 1, 8)
    zg = np.cumsum(rng.uniform(0.2, 0.5, 7))
    deg = order - 1
    cx, cy, cz = rng.normal(size=(3, deg + 1))
    p = lambda x, y, z: np.polyval(cx, x) * np.polyval(cy, y) * np.polyval(cz, z)
    X, Y, Z = np.meshgrid(xg, yg, zg, indexing="ij")
    f = p(X, Y, Z)
    pts = np.stack([rng.uniform(xg[0], xg[-1], 200), rng.uniform(yg[0], yg[-1], 200), rng.uniform(zg[0], zg[-1], 200)], 1)
    val = oracle_dp.bspline3(xg, yg, zg, f, (order, order, order), pts)
    ref = p(pts[:, 0], pts[:, 1], pts[:, 2])
    assert np.max(np.abs(val - ref)) < 1e-11 * max(1.0, np.abs(ref).max())


def test_bspline_range_rules(oracle_dp):
    """db3val returns 0 outside [t(1), t(n+k)] and for y or z at the right end knot, but
    takes the left limit for x at the right end knot (src/bspline/bspline_sub_module.f90)."""
    xg = np.linspace(0, 1, 6)
    f = np.ones((6, 6, 6))
    rnot = 1.0 + 0.1 * (xg[-1] - xg[-2])
    pts = np.array([[-0.01, 0.5, 0.5], [0.5, 0.5, 1.2], [rnot, 0.5, 0.5], [0.5, rnot, 0.5], [0.5, 0.5, rnot], [1.0, 1.0, 1.0]])
    val = oracle_dp.bspline3(xg, xg, xg, f, (4, 4, 4), pts)
    assert val[0] == 0 and val[1] == 0
    assert abs(val[2] - 1.0) < 1e-12  # left limit
    assert val[3] == 0 and val[4] == 0
    assert abs(val[5] - 1.0) < 1e-12


def test_eig3_against_lapack(oracle_dp):
    rng = np.random.default_rng(11)
    for _ in range(200):
        G = rng.normal(size=(3, 3)) * rng.uniform(0.01, 100)
        A = G.T @ G
        assert abs(oracle_dp.eig3_max(A) - np.linalg.eigvalsh(A).max()) <= 1e-13 * np.linalg.eigvalsh(A).max()
    # near-degenerate (two equal largest eigenvalues, as for a rigid rotation)
    th = 0.3
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    D = R - np.eye(3)
    A = D.T @ D
    assert abs(oracle_dp.eig3_max(A) - (2 - 2 * math.cos(th))) < 1e-15


def test_error_latch_and_options(oracle_dp):
    o = oracle_dp
    o.reset()
    o.set_option("INTEGRATOR", 3)
    o.set_option("INTERPOLATOR", 3)
    o.set_param("CFL", 0.9)
    assert o.error() == 0
    o.set_option("NOT_AN_OPTION", 1)
    assert o.error() == 1
    # latched: later calls return immediately
    g = W.abc_grid(4)
    o.init(g.n, g.x, g.y, g.z, g.flag)
    assert o.diagnostic_init(1, 0, 1.0, 0.5) == -1
    o.reset()
    o.set_param("NOT_A_PARAM", 1.0)
    assert o.error() == 1
    o.reset()


def test_update_size_mismatch_latches(oracle_dp):
    o = oracle_dp
    o.reset()
    g = W.abc_grid(6)
    o.init(g.n, g.x, g.y, g.z, g.flag)
    o.n = (5, 6, 6)
    o.update(np.zeros((5, 6, 6)), np.zeros((5, 6, 6)), np.zeros((5, 6, 6)), 0.0)
    assert o.error() == 1
    o.reset()
