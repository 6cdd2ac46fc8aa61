"""Synthetic flows on rectilinear grids, laid out as libcfd2lcs expects them.

Arrays are returned as numpy arrays of shape (ni, nj, nk) in Fortran (i-fastest) order,
the layout `cfd2lcs_init` / `cfd2lcs_update` read.  The flows follow the reference's
example drivers:

* double gyre  -- examples/double_gyre_c.c:164-234 (slip walls, 2-D, time dependent)
* ABC flow     -- examples/abc_flow_c.c:165-223 (triply periodic, cell-centred)
* periodic turbulence -- a seeded divergence-free sum of Fourier modes (k^-5/3 spectrum)
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

LCS_INTERNAL, LCS_INFLOW, LCS_OUTFLOW, LCS_WALL, LCS_SLIP, LCS_2D, LCS_MASK = range(7)


@dataclass
class Grid:
    n: tuple
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    flag: np.ndarray

    @property
    def npts(self) -> int:
        return int(np.prod(self.n))


def _mesh(xl, yl, zl):
    X, Y, Z = np.meshgrid(xl, yl, zl, indexing="ij")
    return np.asfortranarray(X), np.asfortranarray(Y), np.asfortranarray(Z)


# ---------------------------------------------------------------- double gyre
def double_gyre_grid(nx=512, ny=256, lx=2.0, ly=1.0, dtype=np.float64) -> Grid:
    """Node-centred [0,lx]x[0,ly] plane with slip walls (double_gyre_c.c:164-196)."""
    dx = lx / max(nx - 1, 1)
    dy = ly / max(ny - 1, 1)
    xl = np.arange(nx, dtype=np.float64) * dx
    yl = np.arange(ny, dtype=np.float64) * dy
    X, Y, Z = _mesh(xl, yl, np.zeros(1))
    flag = np.full((nx, ny, 1), LCS_INTERNAL, dtype=np.int32, order="F")
    flag[0, :, :] = LCS_SLIP
    flag[-1, :, :] = LCS_SLIP
    flag[:, 0, :] = LCS_SLIP
    flag[:, -1, :] = LCS_SLIP
    return Grid((nx, ny, 1), X.astype(dtype), Y.astype(dtype), Z.astype(dtype), flag)


def double_gyre_velocity(g: Grid, t: float, A=0.1, eps=0.25, omega=2.0 * math.pi / 10.0, dtype=np.float64):
    """u = -pi A sin(pi f) cos(pi y), v = pi A cos(pi f) sin(pi y) df/dx, w = 0 with
    f = eps sin(omega t) x^2 + (1 - 2 eps sin(omega t)) x (double_gyre_c.c:202-234)."""
    x = g.x.astype(np.float64)
    y = g.y.astype(np.float64)
    a = eps * math.sin(omega * t)
    b = 1.0 - 2.0 * eps * math.sin(omega * t)
    f = a * x * x + b * x
    dfdx = 2.0 * a * x + b
    u = -math.pi * A * np.sin(math.pi * f) * np.cos(math.pi * y)
    v = math.pi * A * np.cos(math.pi * f) * np.sin(math.pi * y) * dfdx
    w = np.zeros_like(u)
    return (np.asfortranarray(u.astype(dtype)), np.asfortranarray(v.astype(dtype)), np.asfortranarray(w.astype(dtype)))


# ---------------------------------------------------------------- ABC flow
def abc_grid(n=256, L=2.0 * math.pi, dtype=np.float64, nk=None, nj=None) -> Grid:
    """Cell-centred triply periodic cube, all flags LCS_INTERNAL (abc_flow_c.c:165-194)."""
    nj = n if nj is None else nj
    nk = n if nk is None else nk
    dx, dy, dz = L / n, L / nj, L / nk
    xl = 0.5 * dx + np.arange(n, dtype=np.float64) * dx
    yl = 0.5 * dy + np.arange(nj, dtype=np.float64) * dy
    zl = 0.5 * dz + np.arange(nk, dtype=np.float64) * dz
    X, Y, Z = _mesh(xl, yl, zl)
    flag = np.zeros((n, nj, nk), dtype=np.int32, order="F")
    return Grid((n, nj, nk), X.astype(dtype), Y.astype(dtype), Z.astype(dtype), flag)


def abc_velocity(g: Grid, t: float = 0.0, A=math.sqrt(3.0), B=math.sqrt(2.0), Cc=1.0, D=0.0, dtype=np.float64):
    """u = A sin z + C cos y, v = B sin x + A cos z, w = C sin y + B cos x (abc_flow_c.c:203-223)."""
    x, y, z = (a.astype(np.float64) for a in (g.x, g.y, g.z))
    Ae = A + D * math.sin(t)
    u = Ae * np.sin(z) + Cc * np.cos(y)
    v = B * np.sin(x) + Ae * np.cos(z)
    w = Cc * np.sin(y) + B * np.cos(x)
    return tuple(np.asfortranarray(a.astype(dtype)) for a in (u, v, w))


# ---------------------------------------------------------------- periodic turbulence
@dataclass
class FourierModes:
    k: np.ndarray  # (M,3) integer wavevectors
    a: np.ndarray  # (M,3) amplitudes, a_m . k_m = 0
    phase: np.ndarray
    omega: np.ndarray


def turbulence_modes(nmodes=64, kmin=1, kmax=32, seed=20261203) -> FourierModes:
    """Divergence-free random Fourier modes with |a|^2 ~ E(|k|) dk, E ~ k^-5/3, normalised
    to u_rms = 1; phases U(0,2pi), frequencies U(0,2)."""
    rng = np.random.default_rng(seed)
    ks, amps = [], []
    while len(ks) < nmodes:
        kk = rng.integers(-kmax, kmax + 1, size=3)
        km = float(np.linalg.norm(kk))
        if km < kmin or km > kmax:
            continue
        khat = kk / km
        r = rng.normal(size=3)
        r -= r.dot(khat) * khat
        r /= np.linalg.norm(r)
        ks.append(kk.astype(np.float64))
        amps.append(r * math.sqrt(km ** (-5.0 / 3.0)))
    k = np.array(ks)
    a = np.array(amps)
    rms = math.sqrt(0.5 * float((a * a).sum()) / 3.0)
    a /= rms
    phase = rng.uniform(0.0, 2.0 * math.pi, nmodes)
    omega = rng.uniform(0.0, 2.0, nmodes)
    return FourierModes(k, a, phase, omega)


def turbulence_velocity(g: Grid, t: float, modes: FourierModes, dtype=np.float32):
    """u(x,t) = sum_m a_m cos(k_m . x + omega_m t + phi_m)."""
    x, y, z = (a.astype(np.float64) for a in (g.x, g.y, g.z))
    out = [np.zeros(g.n, dtype=np.float64, order="F") for _ in range(3)]
    for m in range(len(modes.k)):
        arg = modes.k[m, 0] * x + modes.k[m, 1] * y + modes.k[m, 2] * z + modes.omega[m] * t + modes.phase[m]
        c = np.cos(arg)
        for a in range(3):
            out[a] += modes.a[m, a] * c
    return tuple(np.asfortranarray(o.astype(dtype)) for o in out)


def time_at(k: int, dt: float) -> float:
    """Solver time of step k as an exact product (keeps the h-boundary trigger int(t/h)
    deterministic across runs)."""
    return k * dt
