"""Test-only harness: the box FGT as a torch.autograd.Function.

forward runs bfgt_plan_execute (pot = K f on leaf boxes); backward runs the
library's hand-written adjoint bfgt_plan_execute_adjoint (f_bar = K^T pot_bar),
so torch.autograd differentiates through the CUDA transform without tracing
it.  BoxFgtDelta also differentiates with respect to delta: for the kernel
G = exp(-|x|^2/delta), dG/ddelta = |x|^2/delta^2 G = G/delta + (Laplacian G)/4
(the Laplacian acting on the target), so d(K f)/ddelta = K f/delta +
(hess_xx + hess_yy)/4 with the hessian from bfgt_plan_execute_pgh (ifpgh = 3).
Used by the gradient tests only; the library itself has no torch types in its
interface.
"""
from __future__ import annotations

import numpy as np
import torch


class BoxFgt(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fvals, plan):
        fv = fvals.contiguous()
        pot = torch.zeros_like(fv)
        plan.execute(fv, pot)
        ctx.plan = plan
        return pot

    @staticmethod
    def backward(ctx, gpot):
        gf = torch.zeros_like(gpot)
        ctx.plan.execute_adjoint(gpot.contiguous(), gf)
        return gf, None


def boxfgt(fvals, plan):
    return BoxFgt.apply(fvals, plan)


class PlanCache:
    """Plans of one tree, eps and precision, created per delta on demand."""

    def __init__(self, tree, eps, precision):
        self.tree, self.eps, self.precision = tree, eps, precision
        self.plans = {}

    def get(self, delta):
        import heat2d_per_box_b200 as hb
        if delta not in self.plans:
            self.plans[delta] = hb.Plan(self.tree, delta, self.eps, precision=self.precision)
        return self.plans[delta]

    def close(self):
        for p in self.plans.values():
            p.close()
        self.plans = {}


class BoxFgtDelta(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fvals, delta, cache):
        d = float(delta.item())
        plan = cache.get(d)
        fv = fvals.contiguous()
        pot = torch.zeros_like(fv)
        hess = torch.zeros(3 * fv.numel(), dtype=fv.dtype, device=fv.device)
        grad = torch.zeros(2 * fv.numel(), dtype=fv.dtype, device=fv.device)
        plan.execute_pgh(3, fv, pot, grad, hess)
        h = hess.view(-1, 3)  # nd = 1: (point, component)
        ctx.save_for_backward(pot, h[:, 0] + h[:, 2])
        ctx.plan, ctx.delta = plan, d
        return pot

    @staticmethod
    def backward(ctx, gpot):
        pot, lap = ctx.saved_tensors
        gf = torch.zeros_like(gpot)
        ctx.plan.execute_adjoint(gpot.contiguous(), gf)
        dpot = pot / ctx.delta + 0.25 * lap
        gd = torch.sum(gpot * dpot).reshape(1)
        return gf, gd, None


def misfit(fvals, plan, g):
    """J = 0.5 * |K f - g|^2 over the leaf values (g is zero off the leaves)."""
    r = boxfgt(fvals, plan) - g
    return 0.5 * torch.sum(r * r)


def gauss_at_points(pts, gauss):
    """Sum of isotropic Gaussians a exp(-|x-c|^2/w^2) at points (..., 2)."""
    out = np.zeros(pts.shape[:-1])
    for cx, cy, w, a in np.asarray(gauss):
        out += a * np.exp(-((pts[..., 0] - cx) ** 2 + (pts[..., 1] - cy) ** 2) / w ** 2)
    return out
