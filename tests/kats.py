"""Analytic known answers used to pin the oracle and the CUDA path (the reference ships no
tests or golden data, so these are derived from the reference's own semantics)."""
from __future__ import annotations

import math

import numpy as np

from tests import workloads as W


def rk_matrix(A: np.ndarray, dt: float, integrator: int) -> np.ndarray:
    """One integrate_lp step (src/lp_motion_m.f90:129-360) for the steady linear field
    u = A x: the position update is x -> M x.  Stage placement as in the reference (RK3's
    third stage at xn + 2 k2)."""
    I = np.eye(A.shape[0])
    if integrator in (0, 1):  # EULER / TRAPEZOIDAL (velocity at xn)
        return I + dt * A
    if integrator == 2:
        return I + dt * A @ (I + 0.5 * dt * A)
    if integrator == 3:
        K1 = dt * A
        K2 = dt * A @ (I + 0.5 * K1)
        K3 = dt * A @ (I + 2.0 * K2)
        return I + K1 / 6.0 + 2.0 * K2 / 3.0 + K3 / 6.0
    K1 = dt * A
    K2 = dt * A @ (I + 0.5 * K1)
    K3 = dt * A @ (I + 0.5 * K2)
    K4 = dt * A @ (I + K3)
    return I + (K1 + 2 * K2 + 2 * K3 + K4) / 6.0


def rotation_case(n=48, omega=0.5):
    """2-D slip-walled box with a steady solid-body rotation about its centre."""
    g = W.double_gyre_grid(n, n, lx=1.0, ly=1.0)
    xc = yc = 0.5
    u = np.asfortranarray(-omega * (g.y - yc))
    v = np.asfortranarray(omega * (g.x - xc))
    w = np.zeros_like(u)
    A = np.array([[0.0, -omega], [omega, 0.0]])
    return g, (u, v, w), A


def expected_ftle_linear(A2: np.ndarray, dt_sub: float, nsub_total: int, integrator: int, T: float) -> float:
    """FTLE of the reference for a steady linear field: the discrete map after nsub_total
    subcycles is P = M^nsub_total and the reference takes log(sqrt(lmax((P-I)^T (P-I))))/T
    (displacement gradient, src/lcs_m.f90:128-176)."""
    M = rk_matrix(A2, dt_sub, integrator)
    P = np.linalg.matrix_power(M, nsub_total)
    D = P - np.eye(2)
    lam = np.linalg.eigvalsh(D.T @ D).max()
    return math.log(math.sqrt(lam)) / T
