"""torch.autograd.Function over the differentiable step (mf_tangent_mean_force).

    theta = torch.tensor([A, B, n, C, m, mu], dtype=torch.float64, requires_grad=True)
    fc = MeanCuttingForce.apply(theta, ctx, skip_steps, window_steps)
    fc.backward()        # theta.grad = d(mean Fc) / d(A, B, n, C, m, mu)

`ctx` is a product Context holding the scene's state (it is not advanced). The forward pass
runs the FP64 step on dual numbers with no derivative direction; the backward pass runs it once
more with all six parameters' derivatives carried forward together through every step
(mf_tangent_mean_force_all), and returns grad_output times those six derivatives. This module is the only PyTorch in the
package; it imports torch on use.
"""
from __future__ import annotations


PARAMS = ("A", "B", "n", "C", "m", "mu")


def apply_parameters(ctx, theta):
    """Set JC A, B, n, C, m and the tool's friction coefficient from a 6-vector."""
    vals = [float(v) for v in theta]
    phys, corr, joco, tw, tt = ctx.get_constants()
    if joco is None:
        raise ValueError("the context has no Johnson-Cook constants")
    joco.A, joco.B, joco.n, joco.C, joco.m = vals[:5]
    ctx.set_constants(phys, corr, joco, tw, tt)
    tool = ctx.tool_get()
    tool.mu = vals[5]
    ctx.tool_set(tool)


def current_parameters(ctx):
    _, _, joco, _, _ = ctx.get_constants()
    return [joco.A, joco.B, joco.n, joco.C, joco.m, ctx.tool_get().mu]


def _function_class():
    import torch

    class MeanCuttingForce(torch.autograd.Function):
        """Window-averaged cutting force Fc as a function of (A, B, n, C, m, mu)."""

        @staticmethod
        def forward(fctx, theta, ctx, skip_steps, window_steps):
            apply_parameters(ctx, theta.detach().cpu().tolist())
            mean, _ = ctx.tangent_mean_force(skip_steps, window_steps, -1)
            fctx.ctx, fctx.skip, fctx.window = ctx, skip_steps, window_steps
            fctx.save_for_backward(theta)
            return torch.tensor(mean[0], dtype=torch.float64)

        @staticmethod
        def backward(fctx, grad_out):
            (theta,) = fctx.saved_tensors
            apply_parameters(fctx.ctx, theta.detach().cpu().tolist())
            _, dmean = fctx.ctx.tangent_mean_force_all(fctx.skip, fctx.window)
            g = torch.tensor(dmean[:, 0].copy(), dtype=torch.float64) * grad_out
            return g, None, None, None

    return MeanCuttingForce


_CLS = None


def MeanCuttingForce():
    """The autograd Function class (created on first use so that torch loads lazily)."""
    global _CLS
    if _CLS is None:
        _CLS = _function_class()
    return _CLS


def mean_cutting_force(theta, ctx, skip_steps, window_steps):
    return MeanCuttingForce().apply(theta, ctx, skip_steps, window_steps)
