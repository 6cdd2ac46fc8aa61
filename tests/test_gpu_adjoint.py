"""The adjoint (cfd2lcs_adjoint_ftle_c): its forward objective equals the library's own FTLE
frame for h = T, its gradient agrees with central finite differences of that objective along
random directions and with the tangent-linear model (EULER, TRAPEZOIDAL, RK2, RK3 and RK4; LINEAR and
CUBIC interpolation), and it does not depend on the checkpoint interval.  LINEAR also runs on
grids with boundary flags: slip walls on the 2-D double gyre, no-slip walls on a channel,
inflow / outflow / slip / masked nodes on a mixed-boundary box."""
import math

import numpy as np
import pytest

from tests import workloads as W

pytestmark = pytest.mark.gpu


def _levels(n, L, dt, sigma=0.05, seed=7):
    import torch
    g = W.abc_grid(n)
    rng = np.random.default_rng(seed)
    base = W.abc_velocity(g)
    lev = [[], [], []]
    for _ in range(L):
        for c in range(3):
            a = base[c] + sigma * rng.standard_normal(base[c].shape)
            lev[c].append(torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda())
    times = [k * dt for k in range(L)]
    return g, lev, times


def _weight(g):
    import torch
    x, y, z = g.x, g.y, g.z
    box = (x > 0.5 * math.pi) & (x < 1.5 * math.pi) & (y > 0.5 * math.pi) & (y < 1.5 * math.pi) & (z > 0.5 * math.pi) & \
          (z < 1.5 * math.pi)
    w = box.astype(np.float64) / max(int(box.sum()), 1)
    return torch.from_numpy(np.ascontiguousarray(w.ravel(order="F"))).cuda()


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_forward_objective_is_the_library_frame(integrator):
    import libcfd2lcs_b200 as L
    n, nl, dt = 12, 9, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, *_ = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, gradient=False)
    api = L.Cfd2lcs("dp")
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    T = times[-1]
    h = api.diagnostic_init(1, 0, T, T, "b")
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", 1)
    for k in range(nl):
        api.update_device(lev[0][k].data_ptr(), lev[1][k].data_ptr(), lev[2][k].data_ptr(), times[k])
    assert api.error()[0] == 0, api.error()
    ftle = api.ftle(h).ravel(order="F")
    J_lib = float(np.dot(wgt.cpu().numpy(), ftle))
    api.reset()
    assert abs(J - J_lib) <= 1e-12 * max(abs(J_lib), 1e-30), (J, J_lib)


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_gradient_matches_finite_differences(integrator):
    import torch

    import libcfd2lcs_b200 as L
    n, nl, dt = 10, 7, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=2)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(11)
    for _ in range(4):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        eps = 1e-6
        plus = [[lev[c][k] + eps * d[c][k] for k in range(nl)] for c in range(3)]
        minus = [[lev[c][k] - eps * d[c][k] for k in range(nl)] for c in range(3)]
        Jp, *_ = L.adjoint_ftle(g, *plus, times, wgt, integrator=integrator, gradient=False)
        Jm, *_ = L.adjoint_ftle(g, *minus, times, wgt, integrator=integrator, gradient=False)
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), (fd, ad)


def test_checkpoint_interval_does_not_change_the_gradient():
    import torch

    import libcfd2lcs_b200 as L
    g, lev, times = _levels(10, 8, 0.05)
    wgt = _weight(g)
    ref = L.adjoint_ftle(g, *lev, times, wgt, checkpoint_every=100)
    for K in (1, 3):
        out = L.adjoint_ftle(g, *lev, times, wgt, checkpoint_every=K)
        assert out[0] == ref[0]
        for c in range(1, 4):
            for a, b in zip(out[c], ref[c]):
                torch.testing.assert_close(a, b, rtol=1e-12, atol=1e-15)


def test_cubic_adjoint_rejects_walled_grids():
    import torch

    import libcfd2lcs_b200 as L
    g = W.double_gyre_grid(16, 8)
    u = [torch.zeros(16 * 8, dtype=torch.float64, device="cuda") for _ in range(3)]
    with pytest.raises(RuntimeError, match="CUBIC needs"):
        L.adjoint_ftle(g, u, u, u, [0.0, 0.1, 0.2], torch.zeros(16 * 8, dtype=torch.float64, device="cuda"), interpolator=3)


@pytest.mark.parametrize("integrator", [0, 1, 2, 3, 4])
def test_tangent_linear_model_matches_adjoint(integrator):
    """Dot-product test: the forward-mode sweep's dJ along a direction d equals <dJ/du, d> from
    the reverse sweep to rounding (both differentiate the same discrete map with the same
    held-fixed choices), and its J is the adjoint's J."""
    import torch

    import libcfd2lcs_b200 as L
    n, nl, dt = 10, 7, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=3)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(5)
    for _ in range(3):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        Jt, dJ = L.tangent_ftle(g, *lev, times, wgt, *d, integrator=integrator)
        assert Jt == J
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(dJ - ad) <= 1e-11 * max(abs(dJ), abs(ad)), (dJ, ad)


def test_tangent_requires_a_direction():
    import ctypes as C

    import libcfd2lcs_b200 as L
    lib = L.load("dp")
    msg = C.create_string_buffer(256)
    J, dJ = C.c_double(0), C.c_double(0)
    n = np.array([4, 4, 4], dtype=np.int32)
    rc = lib.cfd2lcs_tangent_ftle_c(n.ctypes.data_as(C.c_void_p), None, None, None, 2, 0.5, 2, None, None, None, None, None, None,
                                    None, None, C.byref(J), C.byref(dJ), msg, 256)
    assert rc == 1 and b"direction" in msg.value


# --- CUBIC interpolation (the not-a-knot cubic B-spline, the ABC configuration's interpolator) --

@pytest.mark.parametrize("integrator", [2, 3, 4])
def test_cubic_forward_objective_is_the_library_frame(integrator):
    import libcfd2lcs_b200 as L
    n, nl, dt = 12, 7, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, *_ = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, gradient=False, interpolator=3)
    api = L.Cfd2lcs("dp")
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    T = times[-1]
    h = api.diagnostic_init(1, 0, T, T, "b")
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", 3)
    for k in range(nl):
        api.update_device(lev[0][k].data_ptr(), lev[1][k].data_ptr(), lev[2][k].data_ptr(), times[k])
    assert api.error()[0] == 0, api.error()
    ftle = api.ftle(h).ravel(order="F")
    J_lib = float(np.dot(wgt.cpu().numpy(), ftle))
    api.reset()
    assert abs(J - J_lib) <= 1e-12 * max(abs(J_lib), 1e-30), (J, J_lib)


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_cubic_gradient_matches_finite_differences(integrator):
    import torch

    import libcfd2lcs_b200 as L
    n, nl, dt = 10, 6, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=2, interpolator=3)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(13)
    for _ in range(3):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        eps = 1e-6
        plus = [[lev[c][k] + eps * d[c][k] for k in range(nl)] for c in range(3)]
        minus = [[lev[c][k] - eps * d[c][k] for k in range(nl)] for c in range(3)]
        Jp, *_ = L.adjoint_ftle(g, *plus, times, wgt, integrator=integrator, gradient=False, interpolator=3)
        Jm, *_ = L.adjoint_ftle(g, *minus, times, wgt, integrator=integrator, gradient=False, interpolator=3)
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), (fd, ad)


@pytest.mark.parametrize("integrator", [1, 2, 3, 4])
def test_cubic_tangent_linear_model_matches_adjoint(integrator):
    import torch

    import libcfd2lcs_b200 as L
    n, nl, dt = 10, 6, 0.05
    g, lev, times = _levels(n, nl, dt)
    wgt = _weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=3, interpolator=3)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(17)
    for _ in range(2):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        Jt, dJ = L.tangent_ftle(g, *lev, times, wgt, *d, integrator=integrator, interpolator=3)
        assert Jt == J
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(dJ - ad) <= 1e-11 * max(abs(dJ), abs(ad)), (dJ, ad)


def test_adjoint_rejects_other_interpolators():
    import torch

    import libcfd2lcs_b200 as L
    g, lev, times = _levels(6, 3, 0.05)
    with pytest.raises(RuntimeError, match="LINEAR or CUBIC"):
        L.adjoint_ftle(g, *lev, times, _weight(g), interpolator=2)


# --- LINEAR on grids with boundary flags (walls, slip walls, inflow / outflow, masked nodes) --

def _walled_levels(case, L, dt, sigma=0.02, seed=23):
    import torch

    from tests import scenarios as SC
    n = 16 if case == "dg" else None
    g, vel, _ = SC.make_case(case, n)
    rng = np.random.default_rng(seed)
    lev = [[], [], []]
    for k in range(L):
        comp = vel(k * dt)
        for c in range(3):
            a = np.asarray(comp[c], dtype=np.float64)
            if case == "dg" and c == 2:
                a = np.zeros_like(a)
            else:
                a = a + sigma * rng.standard_normal(a.shape)
            lev[c].append(torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda())
    return g, lev, [k * dt for k in range(L)]


def _random_weight(g, seed=29):
    import torch
    w = np.random.default_rng(seed).uniform(0.5, 1.5, g.x.shape)
    w /= w.sum()
    return torch.from_numpy(np.ascontiguousarray(w.ravel(order="F"))).cuda()


WALLED = [("dg", 0.1), ("channel", 0.05), ("mixed_bc", 0.04)]


@pytest.mark.parametrize("case,dt", WALLED)
@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_walled_forward_objective_is_the_library_frame(case, dt, integrator):
    import libcfd2lcs_b200 as L
    nl = 7
    g, lev, times = _walled_levels(case, nl, dt)
    wgt = _random_weight(g)
    J, *_ = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, gradient=False)
    api = L.Cfd2lcs("dp")
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    T = times[-1]
    h = api.diagnostic_init(1, 0, T, T, "b")
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", 1)
    for k in range(nl):
        api.update_device(lev[0][k].data_ptr(), lev[1][k].data_ptr(), lev[2][k].data_ptr(), times[k])
    assert api.error()[0] == 0, api.error()
    ftle = api.ftle(h).ravel(order="F")
    J_lib = float(np.dot(wgt.cpu().numpy(), ftle))
    api.reset()
    assert abs(J - J_lib) <= 1e-12 * max(abs(J_lib), 1e-30), (J, J_lib)


@pytest.mark.parametrize("case,dt", WALLED)
@pytest.mark.parametrize("integrator", [0, 2, 4])
def test_walled_gradient_matches_finite_differences(case, dt, integrator):
    import torch

    import libcfd2lcs_b200 as L
    nl = 6
    g, lev, times = _walled_levels(case, nl, dt)
    wgt = _random_weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=2)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(31)
    for _ in range(3):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        eps = 1e-7
        plus = [[lev[c][k] + eps * d[c][k] for k in range(nl)] for c in range(3)]
        minus = [[lev[c][k] - eps * d[c][k] for k in range(nl)] for c in range(3)]
        Jp, *_ = L.adjoint_ftle(g, *plus, times, wgt, integrator=integrator, gradient=False)
        Jm, *_ = L.adjoint_ftle(g, *minus, times, wgt, integrator=integrator, gradient=False)
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), (fd, ad)


@pytest.mark.parametrize("case,dt", WALLED)
@pytest.mark.parametrize("integrator", [1, 3])
def test_walled_tangent_linear_model_matches_adjoint(case, dt, integrator):
    import torch

    import libcfd2lcs_b200 as L
    nl = 6
    g, lev, times = _walled_levels(case, nl, dt)
    wgt = _random_weight(g)
    J, gu, gv, gw = L.adjoint_ftle(g, *lev, times, wgt, integrator=integrator, checkpoint_every=4)
    grads = (gu, gv, gw)
    rng = np.random.default_rng(37)
    for _ in range(2):
        d = [[torch.from_numpy(rng.standard_normal(lev[c][k].numel())).cuda() for k in range(nl)] for c in range(3)]
        Jt, dJ = L.tangent_ftle(g, *lev, times, wgt, *d, integrator=integrator)
        assert Jt == J
        ad = sum(float(torch.dot(grads[c][k], d[c][k])) for c in range(3) for k in range(nl))
        assert abs(dJ - ad) <= 1e-11 * max(abs(dJ), abs(ad)), (dJ, ad)
