"""torch.autograd wrapper of the multi-step map and its discrete adjoint.

For gradient checks only (torch.autograd.gradcheck, finite differences):
the forward and backward passes both go through the C ABI
(pamhd_gpu_steps_dt, pamhd_gpu_adjoint) on host tensors, with the dt
schedule given (the adjoint linearises the map on that frozen schedule).
"""
from __future__ import annotations

import numpy as np
import torch


class MHDSteps(torch.autograd.Function):
    """U_N = S_{N-1} o ... o S_0 (U_0) for a pamhd_b200.Context and a fixed dt schedule.

    U0: float64 CPU tensor (8, nz, ny, nx).  Returns U_N of the same shape."""

    @staticmethod
    def forward(ctx, U0, context, dts, every):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        context.set_state(U0.detach().numpy())
        context.steps_dt(dts)
        UN = context.get_state()
        ctx.save_for_backward(U0)
        ctx.context, ctx.dts, ctx.every = context, dts, every
        return torch.from_numpy(UN)

    @staticmethod
    def backward(ctx, grad_out):
        (U0,) = ctx.saved_tensors
        context = ctx.context
        context.set_state(U0.detach().numpy())
        grad, _, _ = context.adjoint(len(ctx.dts), ctx.every, grad_out.detach().contiguous().numpy(),
                                     dt_in=ctx.dts)
        return torch.from_numpy(grad), None, None, None


def steps(U0, context, dts, every=4):
    return MHDSteps.apply(U0, context, dts, every)
