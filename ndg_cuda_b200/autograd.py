"""torch.autograd wrapper of the discrete adjoint (Adjoint2D_t).

`receiver_misfit(adjoint, p0, c, dt, n_steps, targets)` returns the misfit J
as a 0-d tensor whose backward is the library's adjoint sweep: the gradient
with respect to the initial pressure p0 and the per-element wave speed c
comes from ndg_adjoint_backward, not from autograd tracing. Tensors may live
on any device; they are moved to host float64 for the C ABI and the
gradients returned on the inputs' devices and dtypes.
"""
from __future__ import annotations

import numpy as np
import torch


class ReceiverMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p0: torch.Tensor, c: torch.Tensor, adjoint, dt: float, n_steps: int, targets, checkpoint_interval: int):
        p_np = p0.detach().to("cpu", torch.float64).numpy().copy()
        c_np = c.detach().to("cpu", torch.float64).numpy().copy()
        adjoint.set_speed(c_np)
        J, _ = adjoint.forward(p_np, dt, n_steps, targets=targets, checkpoint_interval=checkpoint_interval)
        ctx.adjoint = adjoint
        ctx.inputs = (p_np, c_np, dt, n_steps, targets, checkpoint_interval)
        ctx.serial = adjoint.serial
        ctx.meta = (p0.device, p0.dtype, c.device, c.dtype)
        return torch.tensor(J, dtype=torch.float64, device=p0.device)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        adj = ctx.adjoint
        if adj.serial != ctx.serial:
            # another forward ran on this adjoint since: redo this one
            p_np, c_np, dt, n_steps, targets, interval = ctx.inputs
            adj.set_speed(c_np)
            adj.forward(p_np, dt, n_steps, targets=targets, checkpoint_interval=interval)
        g = adj.backward()
        pd, pt, cd, ct = ctx.meta
        s = float(gJ)
        gp = torch.from_numpy(np.asarray(g["p0"]) * s).to(pd, pt)
        gc = torch.from_numpy(np.asarray(g["c"]) * s).to(cd, ct)
        return gp, gc, None, None, None, None, None


def receiver_misfit(adjoint, p0: torch.Tensor, c: torch.Tensor, dt: float, n_steps: int, targets=None,
                    checkpoint_interval: int = 0) -> torch.Tensor:
    """J(p0, c) = dt/2 sum over steps and receivers of (p_r - target)^2."""
    return ReceiverMisfit.apply(p0, c, adjoint, dt, n_steps, targets, checkpoint_interval)
