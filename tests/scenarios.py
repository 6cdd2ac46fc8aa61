"""Driver loops shared by the parity tests: the same synthetic solver run through the
oracle (CPU restatement) and through libcfd2lcs_b200 (the product), with the calls the
reference's example drivers make (examples/double_gyre_c.c:301-339, abc_flow_c.c:295-333)."""
from __future__ import annotations

import numpy as np

from tests import workloads as W

FTLE_FWD, FTLE_BKWD = 0, 1


def make_case(name: str, n: int | None = None):
    """Returns (grid, velocity(t) callable, dict of run parameters)."""
    if name == "dg":
        g = W.double_gyre_grid(n or 64, (n or 64) // 2)
        return g, (lambda t: W.double_gyre_velocity(g, t)), dict(T=1.5, h=0.15, dt=0.1, steps=40)
    if name == "abc":
        g = W.abc_grid(n or 16)
        vel = W.abc_velocity(g)
        return g, (lambda t: vel), dict(T=1.0, h=0.25, dt=0.05, steps=26)
    if name == "abc_unsteady":
        g = W.abc_grid(n or 12)
        return g, (lambda t: W.abc_velocity(g, t, D=0.3)), dict(T=0.6, h=0.2, dt=0.05, steps=18)
    if name == "channel":
        # periodic x and z, walls in y, non-uniform y spacing: a channel-like grid
        rng = np.random.default_rng(5)
        nx, ny, nz = 10, 8, 6
        yl = np.concatenate([[0.0], np.cumsum(rng.uniform(0.6, 1.4, ny - 1))])
        yl = yl / yl[-1]
        xl = (np.arange(nx) + 0.5) * (2.0 / nx)
        zl = (np.arange(nz) + 0.5) * (1.0 / nz)
        X, Y, Z = np.meshgrid(xl, yl, zl, indexing="ij")
        flag = np.zeros(X.shape, dtype=np.int32)
        flag[:, 0, :] = W.LCS_WALL
        flag[:, -1, :] = W.LCS_WALL
        g = W.Grid((nx, ny, nz), np.asfortranarray(X), np.asfortranarray(Y), np.asfortranarray(Z), np.asfortranarray(flag))

        def vel(t):
            y = g.y
            u = np.asfortranarray(0.6 * 4 * y * (1 - y) + 0.1 * np.sin(2 * np.pi * g.z))
            v = np.asfortranarray(0.05 * np.sin(np.pi * y) * np.cos(np.pi * g.x + t))
            w = np.asfortranarray(0.1 * np.cos(np.pi * g.x) * y * (1 - y))
            return u, v, w

        return g, vel, dict(T=0.6, h=0.2, dt=0.05, steps=16)
    if name == "mixed_bc":
        # inflow / outflow in x, periodic y, slip in z, two masked interior nodes
        nx, ny, nz = 9, 6, 7
        xl, yl, zl = np.arange(nx) * 0.125, (np.arange(ny) + 0.5) / ny, np.arange(nz) * 0.15
        X, Y, Z = np.meshgrid(xl, yl, zl, indexing="ij")
        flag = np.zeros(X.shape, dtype=np.int32)
        flag[0, :, :] = W.LCS_INFLOW
        flag[-1, :, :] = W.LCS_OUTFLOW
        flag[:, :, 0] = W.LCS_SLIP
        flag[:, :, -1] = W.LCS_SLIP
        flag[4, 3, 3] = W.LCS_MASK
        flag[5, 3, 3] = W.LCS_MASK
        g = W.Grid((nx, ny, nz), np.asfortranarray(X), np.asfortranarray(Y), np.asfortranarray(Z), np.asfortranarray(flag))

        def vel(t):
            u = np.asfortranarray(0.4 + 0.1 * np.sin(np.pi * g.z / 0.9) * np.cos(t))
            v = np.asfortranarray(0.08 * np.sin(2 * np.pi * g.x) + 0.05 * np.cos(2 * np.pi * g.y))
            w = np.asfortranarray(0.05 * np.sin(np.pi * g.z / 0.9) * np.sin(2 * np.pi * g.y))
            return u, v, w

        return g, vel, dict(T=0.4, h=0.1, dt=0.05, steps=12)
    if name == "turb":
        # seeded divergence-free Fourier-mode turbulence on a periodic cube (the synthetic
        # turbulence config at a size the oracle runs in seconds; wavenumbers |k| <= 3 so the
        # small grid resolves them)
        g = W.abc_grid(n or 12)
        modes = W.turbulence_modes(nmodes=16, kmin=1, kmax=3, seed=20261203)
        return g, (lambda t: W.turbulence_velocity(g, t, modes, dtype=np.float64)), dict(T=0.2, h=0.05, dt=0.02, steps=16)
    if name in ("curv_box", "curv_periodic", "curv_dg"):
        g = curvilinear_grid(name, n)
        return g, curvilinear_velocity(name, g), dict(T=0.6, h=0.2, dt=0.05, steps=16)
    raise KeyError(name)


def curvilinear_grid(name: str, n: int | None = None):
    """Non-rectilinear grids (the reference's least-squares / TSE_LIMIT path): smooth
    deformations of a box well above check_rectilinear's 1e-4 tolerance.
      curv_box       3-D, slip walls in x and y, walls in z;
      curv_periodic  3-D cube [0, 2 pi)^3 periodic in every direction, deformed by periodic
                     sines (its ghost shifts follow the reference's mirror-minus-image rule);
      curv_dg        2-D (z singleton) box [0, 2] x [0, 1] with slip walls."""
    if name == "curv_box":
        nx, ny, nz = (n or 12), (n or 12) - 2, (n or 12) - 4
        a, b, c = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny), np.linspace(0, 1, nz), indexing="ij")
        X = a + 0.03 * np.sin(2 * np.pi * b) * np.sin(np.pi * c)
        Y = b + 0.03 * np.sin(2 * np.pi * a) * np.sin(np.pi * c)
        Z = c + 0.02 * np.sin(np.pi * a) * np.sin(np.pi * b)
        flag = np.zeros(X.shape, dtype=np.int32)
        flag[0, :, :] = flag[-1, :, :] = W.LCS_SLIP
        flag[:, 0, :] = flag[:, -1, :] = W.LCS_SLIP
        flag[:, :, 0] = flag[:, :, -1] = W.LCS_WALL
    elif name == "curv_periodic":
        m = n or 12
        ln = (np.arange(m) + 0.5) * (2 * np.pi / m)
        a, b, c = np.meshgrid(ln, ln, ln, indexing="ij")
        X = a + 0.08 * np.sin(b) * np.sin(c)
        Y = b + 0.08 * np.sin(c) * np.sin(a)
        Z = c + 0.08 * np.sin(a) * np.sin(b)
        flag = np.zeros(X.shape, dtype=np.int32)
    elif name == "curv_dg":
        nx = n or 32
        ny = nx // 2
        a, b, c = np.meshgrid(np.linspace(0, 2, nx), np.linspace(0, 1, ny), np.zeros(1), indexing="ij")
        X = a + 0.03 * np.sin(np.pi * b) * np.sin(np.pi * a / 2)
        Y = b + 0.02 * np.sin(np.pi * a)
        Z = c
        flag = np.zeros(X.shape, dtype=np.int32)
        flag[0, :, :] = flag[-1, :, :] = W.LCS_SLIP
        flag[:, 0, :] = flag[:, -1, :] = W.LCS_SLIP
    else:
        raise KeyError(name)
    f = np.asfortranarray
    return W.Grid(X.shape, f(X), f(Y), f(Z), f(flag))


def curvilinear_velocity(name: str, g):
    """Smooth unsteady velocity evaluated at the deformed node coordinates."""
    if name == "curv_box":
        def vel(t):
            x, y, z = g.x, g.y, g.z
            u = -0.6 * (y - 0.5) + 0.05 * np.sin(2 * np.pi * z) * np.cos(t)
            v = 0.6 * (x - 0.5) + 0.03 * np.cos(np.pi * z + t)
            w = 0.08 * np.sin(np.pi * x) * np.sin(np.pi * y) * np.cos(2 * t)
            return np.asfortranarray(u), np.asfortranarray(v), np.asfortranarray(w)
        return vel
    if name == "curv_periodic":
        def vel(t):
            x, y, z = g.x, g.y, g.z
            A, B, C = np.sqrt(3.0), np.sqrt(2.0), 1.0
            u = A * np.sin(z) + C * np.cos(y) * (1 + 0.2 * np.sin(t))
            v = B * np.sin(x) + A * np.cos(z)
            w = C * np.sin(y) + B * np.cos(x)
            return np.asfortranarray(u), np.asfortranarray(v), np.asfortranarray(w)
        return vel
    if name == "curv_dg":
        return lambda t: W.double_gyre_velocity(g, t)
    raise KeyError(name)


def run(api, case, directions=(FTLE_BKWD, FTLE_FWD), integrator=2, interpolator=1, cfl=0.5, n=None, steps=None, frames=None):
    """Runs the case through `api` (oracle.Oracle or libcfd2lcs_b200.Cfd2lcs).  Returns the
    handles; results are read from `api` afterwards."""
    g, vel, prm = make_case(case, n)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    handles = [api.diagnostic_init(d, 0, prm["T"], prm["h"], f"d{d}") for d in directions]
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interpolator)
    api.set_param("CFL", cfl)
    nsteps = steps or prm["steps"]
    for k in range(nsteps):
        t = W.time_at(k, prm["dt"])
        u, v, w = vel(t)
        api.update(u, v, w, t)
    return g, handles
