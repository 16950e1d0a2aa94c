"""Gradient and hessian outputs (ifpgh = 2, 3) of the CUDA path against the
oracle's restatement of the reference's g2d_pw2pg / g2d_pw2pgh and
g2d_tens_prod_to_pgloc / _pghloc, through the C ABI.

FP64: pot, grad and hess within 1e-11 relative L2 of the oracle (the same
sums in another order).  Split precision: within min(1e-6, 10 eps) for pot
(its bar) and twice that for the derivatives, whose contractions are the same
split products applied to scaled expansions.
"""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = [("uni3_leg_per", 1e-3, 1e-9), ("uni3_cheb_per", 1e-2, 1e-6), ("uni3_leg_per", 4e-4, 1e-9),
         ("uni3_leg_free", 1e-1, 1e-6), ("ad_leg_per", 1e-4, 1e-6), ("ad_cheb_free", 1e-4, 1e-9),
         ("ad_leg_per", 1e-2, 1e-9), ("lev1_leaf_per", 1e-3, 1e-6), ("ad16_leg_per", 1e-4, 1e-6)]


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def leaf(t, v):
    return np.asarray(v).reshape(t.nboxes, -1)[t.leaves()]


def run_pgh(t, delta, eps, ifpgh, fv=None, nd=1, precision=hb.BFGT_PREC_FP64):
    import torch
    plan = hb.Plan(t, delta, eps, nd=nd, precision=precision)
    f = torch.from_numpy(np.ascontiguousarray(t.fvals if fv is None else fv).reshape(-1)).cuda()
    p = torch.zeros_like(f)
    g = torch.zeros(2 * f.numel(), dtype=f.dtype, device=f.device) if ifpgh >= 2 else None
    h = torch.zeros(3 * f.numel(), dtype=f.dtype, device=f.device) if ifpgh == 3 else None
    plan.execute_pgh(ifpgh, f, p, g, h)
    plan.check()
    out = (p.cpu().numpy(), None if g is None else g.cpu().numpy(), None if h is None else h.cpu().numpy())
    plan.close()
    return out


@pytest.mark.parametrize("name,delta,eps", CASES)
def test_pgh_fp64_matches_oracle(trees, name, delta, eps):
    t = trees[name]
    p, g, h = run_pgh(t, delta, eps, 3)
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 3)
    assert rel_l2(leaf(t, p), leaf(t, rp)) < 1e-11
    assert rel_l2(leaf(t, g), leaf(t, rg)) < 1e-11
    assert rel_l2(leaf(t, h), leaf(t, rh)) < 1e-11
    # pot does not depend on ifpgh
    p1, _, _ = run_pgh(t, delta, eps, 1)
    np.testing.assert_array_equal(p, p1)


def test_pgh_gradient_only_and_densities(trees):
    t = trees["ad_cheb_free"]
    nd = 2
    rng = np.random.default_rng(4)
    fv = np.stack([t.fvals, rng.standard_normal(t.fvals.shape) * (t.nchild() == 0)[:, None]], axis=2)
    fv = np.ascontiguousarray(fv)
    p, g, _ = run_pgh(t, 1e-3, 1e-9, 2, fv=fv, nd=nd)
    rp, rg, _ = oracle.boxfgt_pgh(t, fv, 1e-3, 1e-9, 2, nd=nd)
    assert rel_l2(leaf(t, p), leaf(t, rp)) < 1e-11
    assert rel_l2(leaf(t, g), leaf(t, rg)) < 1e-11


@pytest.mark.parametrize("name,delta,eps", [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9),
                                            ("ad_leg_per", 1e-4, 1e-6), ("uni3_leg_per", 1e-3, 1e-9)])
def test_pgh_split_precision(trees, name, delta, eps):
    t = trees[name]
    p, g, h = run_pgh(t, delta, eps, 3, precision=hb.BFGT_PREC_SPLIT)
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 3)
    assert rel_l2(leaf(t, p), leaf(t, rp)) < min(1e-6, 10 * eps)
    assert rel_l2(leaf(t, g), leaf(t, rg)) < min(2e-6, 20 * eps)
    assert rel_l2(leaf(t, h), leaf(t, rh)) < min(2e-6, 20 * eps)


def test_boxfgt_entry_ifpgh3_host_arrays(trees):
    """The gfortran-ABI boxfgt_ with ifpgh = 3 and host arrays."""
    t = trees["ad_leg_per"]
    delta, eps = 1e-4, 1e-6
    m = t.nboxes * t.npbox
    pot, grad, hess = np.zeros(m), np.zeros(2 * m), np.zeros(3 * m)
    ti = np.zeros(20)
    hb.boxfgt(1, 2, delta, eps, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree, t.itree.copy(),
              t.iptr, t.centers, t.boxsize, np.ascontiguousarray(t.fvals), 3, pot, grad, hess, 0, 0, None, 0, None,
              None, None, ti)
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 3)
    assert rel_l2(leaf(t, pot), leaf(t, rp)) < 1e-11
    assert rel_l2(leaf(t, grad), leaf(t, rg)) < 1e-11
    assert rel_l2(leaf(t, hess), leaf(t, rh)) < 1e-11
