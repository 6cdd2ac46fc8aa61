"""The FTLE adjoint through a torch.autograd.Function in the test harness (tests/autograd_ftle.py):
autograd's gradient of J equals the C ABI's adjoint gradient, composes with a downstream loss
by the chain rule, and agrees with central finite differences of J taken through the same
wrapper along random directions, to 1e-4 of the directional derivative's scale (the error over
the RMS directional derivative, so that directions whose derivative nearly cancels are judged
against the objective's rounding noise rather than their own near-zero value)."""
import math

import numpy as np
import pytest

from tests import workloads as W

pytestmark = pytest.mark.gpu


def _setup(n=10, nl=7, dt=0.05, sigma=0.05, seed=7):
    import torch
    g = W.abc_grid(n)
    rng = np.random.default_rng(seed)
    base = W.abc_velocity(g)
    U = np.stack([np.stack([(base[c] + sigma * rng.standard_normal(base[c].shape)).ravel(order="F") for c in range(3)])
                  for _ in range(nl)])
    x, y, z = g.x, g.y, g.z
    box = (x > 0.5 * math.pi) & (x < 1.5 * math.pi) & (y > 0.5 * math.pi) & (y < 1.5 * math.pi) & (z > 0.5 * math.pi) & \
          (z < 1.5 * math.pi)
    w = box.astype(np.float64).ravel(order="F") / max(int(box.sum()), 1)
    return g, torch.from_numpy(U).cuda(), [k * dt for k in range(nl)], torch.from_numpy(w).cuda()


def test_autograd_gradient_is_the_adjoint():
    import torch

    import libcfd2lcs_b200 as L
    from tests.autograd_ftle import FtleObjective
    g, U, times, w = _setup()
    U.requires_grad_(True)
    J = FtleObjective.apply(U, g, times, w, 2, 3)
    (G,) = torch.autograd.grad(J, U)
    nl = U.shape[0]
    Jc, gu, gv, gw = L.adjoint_ftle(g, [U[k, 0].detach().contiguous() for k in range(nl)],
                                    [U[k, 1].detach().contiguous() for k in range(nl)],
                                    [U[k, 2].detach().contiguous() for k in range(nl)], times, w, integrator=2, checkpoint_every=3)
    # (the reverse sweep scatters with atomic adds, so two runs agree to rounding, not bitwise)
    assert abs(float(J) - Jc) <= 1e-12 * abs(Jc)
    ref = torch.stack([torch.stack([gu[k], gv[k], gw[k]]) for k in range(nl)])
    assert torch.allclose(G, ref, rtol=1e-10, atol=1e-12 * float(ref.abs().max()))
    # chain rule through a downstream loss: d(J^2)/dU = 2 J dJ/dU
    U.grad = None
    (FtleObjective.apply(U, g, times, w, 2, 3) ** 2).backward()
    assert torch.allclose(U.grad, 2.0 * J.detach() * ref, rtol=1e-10, atol=1e-12 * float(ref.abs().max()))


def test_autograd_matches_finite_differences():
    import torch

    from tests.autograd_ftle import FtleObjective
    g, U, times, w = _setup()
    U.requires_grad_(True)
    J = FtleObjective.apply(U, g, times, w, 2, 3)
    J.backward()
    rng = np.random.default_rng(11)
    eps = 1e-6
    fds, ads = [], []
    with torch.no_grad():
        for _ in range(8):
            d = torch.from_numpy(rng.standard_normal(tuple(U.shape))).cuda()
            Jp = float(FtleObjective.apply(U + eps * d, g, times, w, 2, 3))
            Jm = float(FtleObjective.apply(U - eps * d, g, times, w, 2, 3))
            fds.append((Jp - Jm) / (2 * eps))
            ads.append(float((U.grad * d).sum()))
    fds, ads = np.array(fds), np.array(ads)
    scale = float(np.sqrt(np.mean(ads ** 2)))
    err = np.abs(fds - ads) / scale
    assert float(err.max()) <= 1e-4, (err, fds, ads)
