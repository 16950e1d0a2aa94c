"""The transposed transform (bfgt_plan_execute_adjoint) on the GPU.

For pot = K f (bfgt_plan_execute, leaf boxes) the adjoint must satisfy
sum(g * K f) = sum(f * K^T g) over leaf values.  Checked three ways:
  * against the GPU forward transform, every regime (A periodic Fourier,
    B plane waves + near field, C near field only), free and periodic,
    Legendre and Chebyshev leaves, a periodic level-1 image, nd > 1;
  * against the oracle's forward transform (the CPU restatement of the
    reference), so that the identity pins K^T to the reference's K;
  * as the gradient of J = 0.5 |K f - g|^2 through a torch.autograd.Function
    whose backward is the adjoint, against central differences (step 1e-6)
    along 100 random directions on an order-16 adaptive tree at delta = 1e-3.
Tolerances: FP64 plans to 1e-12 (relative to |K f| |g|); the split-precision
adjoint to 1e-6 relative L2 against the FP64 adjoint.
"""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

from conftest import gauss_sum

pytestmark = pytest.mark.gpu

CASES = [
    ("uni3_leg_per", 1e-3, 1e-9),    # regime B
    ("uni3_cheb_per", 1e-2, 1e-6),   # regime A (periodic Fourier)
    ("uni3_leg_per", 4e-4, 1e-9),    # regime C (near field only)
    ("uni3_leg_free", 1e-1, 1e-6),   # free space, cutoff at the root
    ("ad_leg_per", 1e-4, 1e-6),
    ("ad_cheb_free", 1e-4, 1e-9),
    ("ad_leg_per", 1e-2, 1e-9),      # odd npw
    ("lev1_leaf_per", 1e-3, 1e-6),   # periodic level-1 images
    ("lev1_leaf_per", 2e-2, 1e-9),
    ("ad16_leg_per", 1e-4, 1e-6),
]


def leaf_random(t, nd, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((t.nboxes, t.npbox, nd))
    lv = t.leaves()
    x[lv] = rng.standard_normal((len(lv), t.npbox, nd))
    return x


def fwd_adj(t, delta, eps, f, g, nd=1, precision=hb.BFGT_PREC_FP64):
    import torch
    plan = hb.Plan(t, delta, eps, nd=nd, precision=precision)
    df = torch.from_numpy(f.reshape(-1).copy()).cuda()
    dg = torch.from_numpy(g.reshape(-1).copy()).cuda()
    kf = torch.zeros_like(df)
    ktg = torch.zeros_like(dg)
    plan.execute(df, kf)
    plan.execute_adjoint(dg, ktg)
    plan.check()
    out = kf.cpu().numpy(), ktg.cpu().numpy()
    plan.close()
    return out


@pytest.mark.parametrize("name,delta,eps", CASES)
def test_adjoint_identity_fp64(trees, name, delta, eps):
    t = trees[name]
    f, g = leaf_random(t, 1, 1), leaf_random(t, 1, 2)
    kf, ktg = fwd_adj(t, delta, eps, f, g)
    a, b = np.dot(kf, g.reshape(-1)), np.dot(f.reshape(-1), ktg)
    scale = np.linalg.norm(kf) * np.linalg.norm(g)
    assert abs(a - b) <= 1e-12 * scale, (a, b, scale)
    # nothing is written off the leaves
    nonleaf = np.nonzero(t.nchild() > 0)[0]
    assert not np.any(ktg.reshape(t.nboxes, -1)[nonleaf])


@pytest.mark.parametrize("name,delta,eps", [CASES[0], CASES[1], CASES[2], CASES[5], CASES[7]])
def test_adjoint_against_oracle_forward(trees, name, delta, eps):
    t = trees[name]
    for s in range(3):
        f, g = leaf_random(t, 1, 10 + s), leaf_random(t, 1, 20 + s)
        _, ktg = fwd_adj(t, delta, eps, f, g)
        kf_ref = oracle.boxfgt(t, f.reshape(t.nboxes, t.npbox), delta, eps).reshape(-1)
        a, b = np.dot(kf_ref, g.reshape(-1)), np.dot(f.reshape(-1), ktg)
        assert abs(a - b) <= 1e-11 * np.linalg.norm(kf_ref) * np.linalg.norm(g), (a, b)


def test_adjoint_multiple_densities(trees):
    t = trees["ad_cheb_free"]
    nd = 3
    f, g = leaf_random(t, nd, 3), leaf_random(t, nd, 4)
    kf, ktg = fwd_adj(t, 1e-4, 1e-6, f, g, nd=nd)
    for d in range(nd):
        gd = np.zeros_like(g)
        gd[:, :, d] = g[:, :, d]
        fd = np.zeros_like(f)
        fd[:, :, d] = f[:, :, d]
        a = np.dot(kf, gd.reshape(-1))
        b = np.dot(fd.reshape(-1), ktg)
        assert abs(a - b) <= 1e-12 * np.linalg.norm(kf) * np.linalg.norm(g)


def test_adjoint_host_entry_matches_device(trees):
    t = trees["ad_leg_per"]
    g = leaf_random(t, 1, 9).reshape(-1)
    _, ktg = fwd_adj(t, 1e-4, 1e-6, np.zeros_like(g), g)
    plan = hb.Plan(t, 1e-4, 1e-6)
    acc = np.zeros_like(g)
    plan.execute_adjoint_host(g, acc)
    plan.close()
    np.testing.assert_allclose(acc, ktg, rtol=0, atol=1e-14 * np.abs(ktg).max())


@pytest.mark.parametrize("name,delta,eps", [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9),
                                            ("ad16_leg_per", 1e-2, 1e-6), ("ad_leg_per", 1e-4, 1e-6),
                                            ("uni3_leg_per", 1e-3, 1e-9)])
def test_adjoint_split_precision(trees, name, delta, eps):
    t = trees[name]
    f, g = leaf_random(t, 1, 5), leaf_random(t, 1, 6)
    kf, ktg64 = fwd_adj(t, delta, eps, f, g)
    _, ktg = fwd_adj(t, delta, eps, f, g, precision=hb.BFGT_PREC_SPLIT)
    err = np.linalg.norm(ktg - ktg64) / np.linalg.norm(ktg64)
    bar = min(1e-6, 10 * eps)
    assert err <= bar, err
    a, b = np.dot(kf, g.reshape(-1)), np.dot(f.reshape(-1), ktg)
    assert abs(a - b) <= bar * np.linalg.norm(kf) * np.linalg.norm(g)


def _c4_tree():
    """Order-16 adaptive periodic tree with the benchmark density statistics
    (20 Gaussians, widths log-uniform in [1e-3, 1e-2], N(0,1) amplitudes),
    uniform to level 5, refined to a 1e-10 Legendre tail, max level 9."""
    g = gauss_sum(2, 20, 1e-3, 1e-2, amp="normal", log_width=True)
    return hb.build_adaptive(g, norder=16, ipoly=0, iperiod=1, eps=1e-10, minlev=5, maxlev=9)


def _c2_bench_tree():
    """The benchmark's adaptive order-16 tree statistics at full size: 20
    Gaussians (widths log-uniform in [1e-3, 1e-2], N(0,1) amplitudes), uniform
    to level 8, refined to a 1e-10 Legendre tail, max level 12 (~65k leaves)."""
    g = gauss_sum(2, 20, 1e-3, 1e-2, amp="normal", log_width=True)
    return hb.build_adaptive(g, norder=16, ipoly=0, iperiod=1, eps=1e-10, minlev=8, maxlev=12)


def _gradient_check(t, precision, tol, ndir=100):
    """dJ/df through autograd (backward = the adjoint) vs central differences of
    the FP64 transform, h = 1e-6, ndir random leaf directions drawn on the
    device (seed 7)."""
    import torch
    from fgt_autograd import boxfgt, gauss_at_points, misfit

    delta, eps = 1e-3, 1e-9
    lv = t.leaves()
    gpar = gauss_sum(3, 20, 1e-3, 1e-2, amp="normal", log_width=True)
    gt = np.zeros((t.nboxes, t.npbox))
    gt[lv] = gauss_at_points(t.grid_points(lv), gpar)
    f0 = np.zeros((t.nboxes, t.npbox))
    f0[lv] = t.fvals[lv]
    dev = torch.device("cuda")
    g = torch.from_numpy(gt.reshape(-1)).to(dev)
    plan = hb.Plan(t, delta, eps, precision=precision)
    f = torch.from_numpy(f0.reshape(-1)).to(dev).requires_grad_(True)
    J = misfit(f, plan, g)
    J.backward()
    plan.check()
    grad = f.grad.detach()
    ref = hb.Plan(t, delta, eps, precision=hb.BFGT_PREC_FP64)
    gen = torch.Generator(device=dev)
    gen.manual_seed(7)
    mask = torch.zeros(t.nboxes, t.npbox, dtype=torch.float64, device=dev)
    mask[torch.from_numpy(lv).to(dev)] = 1.0
    mask = mask.reshape(-1)
    h = 1e-6
    fd, an = [], []
    with torch.no_grad():
        for _ in range(ndir):
            vt = torch.randn(mask.shape, generator=gen, dtype=torch.float64, device=dev) * mask
            rp = boxfgt(f.detach() + h * vt, ref) - g
            rm = boxfgt(f.detach() - h * vt, ref) - g
            fd.append((0.5 * torch.sum((rp - rm) * (rp + rm))).item() / (2 * h))
            an.append(torch.dot(grad, vt).item())
    plan.close()
    ref.close()
    fd, an = np.array(fd), np.array(an)
    err = np.linalg.norm(fd - an) / np.linalg.norm(fd)
    assert err <= tol, err


@pytest.mark.parametrize("precision,tol", [(hb.BFGT_PREC_FP64, 1e-7), (hb.BFGT_PREC_SPLIT, 1e-6)])
def test_gradient_on_the_benchmark_tree(precision, tol):
    """Configuration C4 at its size: the gradient check on the benchmark's
    adaptive order-16 tree (65k leaves, 16.8 M leaf values), delta = 1e-3."""
    _gradient_check(_c2_bench_tree(), precision, tol)


@pytest.mark.parametrize("precision,tol", [(hb.BFGT_PREC_FP64, 1e-7), (hb.BFGT_PREC_SPLIT, 1e-6)])
def test_gradient_matches_central_differences(precision, tol):
    """dJ/df through autograd (backward = the adjoint) vs central differences of
    the FP64 transform, h = 1e-6, 100 random directions (seed 7)."""
    import torch
    from fgt_autograd import boxfgt, gauss_at_points, misfit

    t = _c4_tree()
    delta, eps = 1e-3, 1e-9
    lv = t.leaves()
    gpar = gauss_sum(3, 20, 1e-3, 1e-2, amp="normal", log_width=True)
    gt = np.zeros((t.nboxes, t.npbox))
    gt[lv] = gauss_at_points(t.grid_points(lv), gpar)
    f0 = np.zeros((t.nboxes, t.npbox))
    f0[lv] = t.fvals[lv]
    dev = torch.device("cuda")
    g = torch.from_numpy(gt.reshape(-1)).to(dev)
    plan = hb.Plan(t, delta, eps, precision=precision)
    f = torch.from_numpy(f0.reshape(-1)).to(dev).requires_grad_(True)
    J = misfit(f, plan, g)
    J.backward()
    plan.check()
    grad = f.grad.detach()
    ref = hb.Plan(t, delta, eps, precision=hb.BFGT_PREC_FP64)
    rng = np.random.default_rng(7)
    h = 1e-6
    fd, an = [], []
    with torch.no_grad():
        for _ in range(100):
            v = np.zeros_like(f0)
            v[lv] = rng.standard_normal((len(lv), t.npbox))
            vt = torch.from_numpy(v.reshape(-1)).to(dev)
            rp = boxfgt(f.detach() + h * vt, ref) - g
            rm = boxfgt(f.detach() - h * vt, ref) - g
            # J(f+hv) - J(f-hv) = 0.5 sum (rp - rm)(rp + rm), summed elementwise
            # so that the two large sums do not cancel
            fd.append((0.5 * torch.sum((rp - rm) * (rp + rm))).item() / (2 * h))
            an.append(torch.dot(grad, vt).item())
    plan.close()
    ref.close()
    fd, an = np.array(fd), np.array(an)
    err = np.linalg.norm(fd - an) / np.linalg.norm(fd)
    assert err <= tol, err


@pytest.mark.parametrize("precision", [hb.BFGT_PREC_FP64, hb.BFGT_PREC_SPLIT])
def test_delta_gradient_matches_central_differences(precision, tol=1e-6):
    """dJ/ddelta through autograd (the hessian identity of fgt_autograd) vs
    central differences of the FP64 transform in delta, relative step 1e-6, on
    the same order-16 tree at delta = 1e-3 (eps = 1e-9).  The identity is the
    derivative of the exact Gaussian kernel; the differences see the discrete
    transform, whose approximation error also moves with delta, so the two
    agree to the transform's accuracy (about 2e-7 here), within the 1e-6 bar."""
    import torch
    from fgt_autograd import BoxFgtDelta, PlanCache, gauss_at_points

    t = _c4_tree()
    delta, eps = 1e-3, 1e-9
    lv = t.leaves()
    gpar = gauss_sum(3, 20, 1e-3, 1e-2, amp="normal", log_width=True)
    gt = np.zeros((t.nboxes, t.npbox))
    gt[lv] = gauss_at_points(t.grid_points(lv), gpar)
    f0 = np.zeros((t.nboxes, t.npbox))
    f0[lv] = t.fvals[lv]
    dev = torch.device("cuda")
    g = torch.from_numpy(gt.reshape(-1)).to(dev)
    f = torch.from_numpy(f0.reshape(-1)).to(dev)
    cache = PlanCache(t, eps, precision)
    d = torch.tensor([delta], dtype=torch.float64, device=dev, requires_grad=True)
    r = BoxFgtDelta.apply(f, d, cache) - g
    J = 0.5 * torch.sum(r * r)
    J.backward()
    an = d.grad.item()
    ref = PlanCache(t, eps, hb.BFGT_PREC_FP64)
    h = 1e-6 * delta
    with torch.no_grad():
        rp = BoxFgtDelta.apply(f, torch.tensor([delta + h], dtype=torch.float64, device=dev), ref) - g
        rm = BoxFgtDelta.apply(f, torch.tensor([delta - h], dtype=torch.float64, device=dev), ref) - g
        fd = (0.5 * torch.sum((rp - rm) * (rp + rm))).item() / (2 * h)
    for pl in list(cache.plans.values()) + list(ref.plans.values()):
        assert pl.info()["npw"] == next(iter(ref.plans.values())).info()["npw"]
    cache.close()
    ref.close()
    assert abs(fd - an) <= tol * abs(fd), (fd, an)
