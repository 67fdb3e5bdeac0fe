"""d(plastic strain)/d(initial positions, external stress) as a
torch.autograd.Function.

The forward is the engine's fixed-step replay of recorded accepted steps
(d4_replay), the backward its hand-written adjoint (d4_adjoint: checkpointed
positions, the step's LU factors reused for the transposed solves).  Step sizes
are constants of the function: record them with ``Engine.record_steps`` during
an adaptive run, then differentiate the replay of that sequence.  PyTorch only
carries the values and gradients across this boundary; all arithmetic runs in
libd4core.so.
"""
import numpy as np
import torch


class StrainFunction(torch.autograd.Function):
    """strain = StrainFunction.apply(x0, tau0, engine, t0s, hs, checkpoint_every)

    x0: float64 tensor of n positions (internal order); tau0: float64 scalar
    tensor (the protocol's initial external stress).  Returns a float64 scalar."""

    @staticmethod
    def forward(ctx, x0, tau0, engine, t0s, hs, checkpoint_every=20):
        xs = x0.detach().cpu().numpy().astype(np.float64)
        tv = float(tau0.detach().cpu())
        strain, _ = engine.replay(xs, t0s, hs, tau0=tv)
        ctx.engine, ctx.t0s, ctx.hs, ctx.k = engine, t0s, hs, checkpoint_every
        ctx.xs, ctx.tv = xs, tv
        ctx.dev = x0.device
        return torch.tensor(strain, dtype=torch.float64, device=x0.device)

    @staticmethod
    def backward(ctx, grad_out):
        _, g, gt = ctx.engine.adjoint(ctx.xs, ctx.t0s, ctx.hs, ctx.k, tau0=ctx.tv)
        go = float(grad_out.detach().cpu())
        gx = torch.as_tensor(g * go, dtype=torch.float64, device=ctx.dev)
        gtau = torch.tensor(gt * go, dtype=torch.float64, device=ctx.dev)
        return gx, gtau, None, None, None, None


def strain(x0, tau0, engine, t0s, hs, checkpoint_every=20):
    return StrainFunction.apply(x0, tau0, engine, t0s, hs, checkpoint_every)
