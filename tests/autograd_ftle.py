"""torch.autograd wrapper of the library's FTLE adjoint, for the Python test harness only (the
library's interface is the C ABI: cfd2lcs_adjoint_ftle_c, cfd2lcs_tangent_ftle_c).

FtleObjective.apply(U, grid, times, weight, integrator, checkpoint_every) returns the scalar
J = sum_x weight(x) FTLE(x) of the backward flow map over all velocity levels, as a function of
the gridded velocity U -- a CUDA float64 tensor of shape (levels, 3, n[0]*n[1]*n[2]), i fastest
-- so that J.backward() (or torch.autograd.grad) delivers dJ/dU through the hand-written
reverse sweep.  The forward call runs the adjoint once and keeps the gradient for backward.
"""
import torch

import libcfd2lcs_b200 as L


class FtleObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, grid, times, weight, integrator=2, checkpoint_every=20):
        nl = U.shape[0]
        us = [U[k, 0].contiguous() for k in range(nl)]
        vs = [U[k, 1].contiguous() for k in range(nl)]
        ws = [U[k, 2].contiguous() for k in range(nl)]
        need = U.requires_grad
        J, gu, gv, gw = L.adjoint_ftle(grid, us, vs, ws, times, weight, integrator=integrator, checkpoint_every=checkpoint_every,
                                       gradient=need)
        if need:
            ctx.save_for_backward(torch.stack([torch.stack([gu[k], gv[k], gw[k]]) for k in range(nl)]))
        return torch.tensor(J, dtype=torch.float64, device=U.device)

    @staticmethod
    def backward(ctx, gJ):
        (G,) = ctx.saved_tensors
        return gJ * G, None, None, None, None, None
