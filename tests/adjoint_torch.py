"""torch.autograd.Function wrappers of the adjoint gradient, for the tests only.

The product computes gradients through its C ABI (tw_adjoint_gradient, tw_adjoint_gradient_revolve);
these wrappers let the tests state the finite-difference and dot-product checks as ordinary
autograd computations (torch.autograd.grad on a scalar misfit, vector-Jacobian products of the
traces), so that the adjoint is exercised exactly as a PyTorch caller would use it.

* Misfit.apply(rho, vp, vs, runner): J = 1/2 sum (traces - obs)^2 of the padded node model; the
  backward pass returns dJ/d(rho, vp, vs) from one adjoint call. `runner(rho, vp, vs)` returns
  (J, {"rho": ..., "vp": ..., "vs": ...}) as numpy arrays.
* Traces.apply(x0, ..., x4, runner): the traces of a run started from the initial fields x (no
  source), a linear map L; the backward pass returns L^T y for the incoming y, computed by the
  adjoint with the observed traces set to L x - y (its residual is then y).
"""
import numpy as np
import torch


class Misfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, vp, vs, runner):
        J, g = runner(rho.detach().numpy(), vp.detach().numpy(), vs.detach().numpy())
        ctx.save_for_backward(*(torch.from_numpy(np.ascontiguousarray(g[k])) for k in ("rho", "vp", "vs")))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        g_rho, g_vp, g_vs = ctx.saved_tensors
        return gJ * g_rho, gJ * g_vp, gJ * g_vs, None


class Traces(torch.autograd.Function):
    """runner.forward(x) -> traces; runner.transpose(x, obs) -> the initial-state gradient (5 arrays)
    of 1/2 |L x - obs|^2."""

    @staticmethod
    def forward(ctx, x0, x1, x2, x3, x4, runner):
        xs = [t.detach().numpy() for t in (x0, x1, x2, x3, x4)]
        d = runner.forward(xs)
        ctx.runner = runner
        ctx.xs = xs
        ctx.d = d
        return torch.from_numpy(d)

    @staticmethod
    def backward(ctx, y):
        g = ctx.runner.transpose(ctx.xs, ctx.d - y.detach().numpy())
        return (*(torch.from_numpy(np.ascontiguousarray(a)) for a in g), None)
