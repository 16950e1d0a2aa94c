"""Test-only harness: the box FGT as a torch.autograd.Function.

forward runs bfgt_plan_execute (pot = K f on leaf boxes); backward runs the
library's hand-written adjoint bfgt_plan_execute_adjoint (f_bar = K^T pot_bar),
so torch.autograd differentiates through the CUDA transform without tracing
it.  Used by the gradient tests only; the library itself has no torch types
in its interface.
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
