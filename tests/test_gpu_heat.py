"""Configuration C5 on a fixed tree: a time-stepped periodic reaction-diffusion
solve through the box FGT (tests/heat_solver.py), every step one batch of 5
transforms replayed as one CUDA graph, and the gradient of a final-time misfit
with respect to the initial condition by checkpointed adjoint stepping.

Manufactured solution u = sin(2 pi x) cos(2 pi y) exp(-t) (the reference's
solver test hpots/test_forcing_adap1.f:86-112 uses the same field) with the
source S = (8 pi^2 - 1) u + u^3 that makes u_t = Laplacian(u) + S - u^3 hold.
dt = 1e-3, 200 steps, order-8 Legendre leaves on a uniform level-4 periodic
tree, and at the configuration's size on an adaptive tree of 6,970 leaves
(levels 6-8) refined around 10 Gaussians of width 0.02.  The tree stays fixed:
refinement and coarsening between steps are the solver's own tree work
(vol_tree_adap_fv), which this library does not rebuild.
"""
import math

import numpy as np
import pytest

import heat2d_per_box_b200 as hb

pytestmark = pytest.mark.gpu

DT, NSTEPS = 1e-3, 200


def c5_tree():
    """Adaptive periodic order-8 tree of the configuration's size: refined to a
    1e-10 tail around 10 Gaussians of width 0.02 (seed 5), levels 6 to 8."""
    rng = np.random.default_rng(5)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (10, 2)), np.full(10, 0.02), np.ones(10))
    return hb.build_adaptive(g, norder=8, ipoly=0, iperiod=1, eps=1e-10, minlev=6, maxlev=9)


def setup(precision, eps, tree=None):
    import torch
    from heat_solver import HeatStepper
    g = hb.gauss_params(np.zeros((1, 2)), np.ones(1), np.zeros(1))
    t = hb.build_uniform(4, g, norder=8, ipoly=0, iperiod=1) if tree is None else tree
    lv = t.leaves()
    xy = t.grid_points(lv)
    A = np.zeros((t.nboxes, t.npbox))
    A[lv] = np.sin(2 * np.pi * xy[..., 0]) * np.cos(2 * np.pi * xy[..., 1])
    A = torch.from_numpy(A.reshape(-1)).cuda()
    c = 8 * math.pi ** 2 - 1

    def source(tt):
        return c * A * math.exp(-tt) + A ** 3 * math.exp(-3 * tt)

    st = HeatStepper(t, DT, eps, precision, source)
    hist = [c * A * math.exp(j * DT) for j in (1, 2, 3)]   # F = S - u^3 on the exact solution
    return st, A, hist


@pytest.mark.parametrize("precision,tol", [(hb.BFGT_PREC_FP64, 1e-7), (hb.BFGT_PREC_SPLIT, 2e-5)])
def test_heat_stepping_matches_exact_solution(precision, tol):
    st, A, hist = setup(precision, 1e-9 if precision == hb.BFGT_PREC_FP64 else 1e-6)
    uN = st.run(A.clone(), hist, NSTEPS)
    st.batch.check()
    exact = A * math.exp(-NSTEPS * DT)
    err = (uN - exact).norm().item() / exact.norm().item()
    st.close()
    assert err < tol, err


@pytest.mark.parametrize("precision,tol", [(hb.BFGT_PREC_FP64, 1e-7), (hb.BFGT_PREC_SPLIT, 2e-5)])
def test_heat_stepping_at_configuration_size(precision, tol):
    t = c5_tree()
    assert 4000 <= len(t.leaves()) <= 16000
    st, A, hist = setup(precision, 1e-9 if precision == hb.BFGT_PREC_FP64 else 1e-6, tree=t)
    uN = st.run(A.clone(), hist, NSTEPS)
    st.batch.check()
    exact = A * math.exp(-NSTEPS * DT)
    err = (uN - exact).norm().item() / exact.norm().item()
    st.close()
    assert err < tol, err


@pytest.mark.parametrize("size", ["level4", "c5"])
def test_heat_gradient_checkpointed_adjoint_vs_central_differences(size):
    import torch
    st, A, hist = setup(hb.BFGT_PREC_FP64, 1e-9, tree=c5_tree() if size == "c5" else None)
    rng = np.random.default_rng(7)
    leaf = st.leaf.cpu().numpy()
    g = torch.from_numpy(0.5 * rng.standard_normal(leaf.size) * leaf).cuda()
    u0 = A.clone()
    grad = st.gradient(u0, hist, NSTEPS, g, ckpt=20)
    # h = 1e-4: the cubic term keeps the O(h^2) error below 1e-10 here, while
    # at 1e-6 rounding in the 200-step differences reaches 1e-6
    h = 1e-4
    fd, an = [], []
    for _ in range(4):
        v = torch.from_numpy(rng.standard_normal(leaf.size) * leaf).cuda()
        up = st.run(u0 + h * v, hist, NSTEPS)
        um = st.run(u0 - h * v, hist, NSTEPS)
        fd.append((0.5 * torch.sum((up - um) * (up + um - 2 * g))).item() / (2 * h))
        an.append(torch.dot(grad, v).item())
    st.close()
    fd, an = np.array(fd), np.array(an)
    err = np.linalg.norm(fd - an) / np.linalg.norm(fd)
    assert err < 1e-6, (fd, an, err)
