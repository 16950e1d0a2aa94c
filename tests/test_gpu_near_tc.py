"""The near field (step 6: g2d_tens_prod_to_potloc, bfgt/bfgt_local.f:315-375,
loop boxfgt.f:915-1071) of split-precision plans on the tensor cores: regime C
trees (small delta, every interaction in the near field), orders 8 and 16,
periodic and free space, Legendre and Chebyshev, leaves next to periodic
level-1 images.  Bar: min(1e-6, 10 eps) relative L2 against the oracle.  The
FP64 plan of the same tree runs the FP64 near-field kernel, so the two results
differ (in the last bits) when the tensor-core kernel ran.  Each density of
an nd = 3 plan equals, bit for bit, the nd = 1 transform of it."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run(t, delta, eps, precision, f=None, nd=1):
    import torch
    f = t.fvals if f is None else f
    plan = hb.Plan(t, delta, eps, nd=nd, precision=precision)
    fd = torch.from_numpy(np.ascontiguousarray(f).reshape(-1)).cuda()
    p = torch.zeros_like(fd)
    plan.execute(fd, p)
    plan.check()
    info = plan.info()
    plan.close()
    return p.cpu().numpy(), info


CASES = [("uni3_leg_per", 1e-5, 1e-6), ("uni3_cheb_per", 3e-5, 1e-6), ("uni3_leg_free", 1e-5, 1e-6),
         ("ad_leg_per", 1e-5, 1e-6), ("ad_cheb_free", 3e-5, 1e-6), ("ad16_leg_per", 1e-5, 1e-6),
         ("ad16_leg_per", 3e-6, 1e-7), ("lev1_leaf_per", 1e-4, 1e-6), ("ad_leg_per", 1e-4, 1e-6)]


@pytest.mark.parametrize("name,delta,eps", CASES)
def test_near_field_on_tensor_cores_matches_oracle(trees, name, delta, eps):
    t = trees[name]
    lv = t.leaves()
    p, info = run(t, delta, eps, hb.BFGT_PREC_SPLIT)
    assert info["nnear_pairs"] > 0
    ref = oracle.boxfgt(t, t.fvals, delta, eps).reshape(t.nboxes, -1)[lv]
    got = p.reshape(t.nboxes, -1)[lv]
    assert rel_l2(got, ref) < min(1e-6, 10 * eps)
    q, _ = run(t, delta, eps, hb.BFGT_PREC_FP64)
    assert rel_l2(q.reshape(t.nboxes, -1)[lv], ref) < 1e-11
    assert not np.array_equal(p, q)  # the split plan's near field is not the FP64 kernel's
    # non-leaf boxes are not written
    nl = t.nchild() > 0
    assert not p.reshape(t.nboxes, -1)[nl].any()


@pytest.mark.parametrize("name,delta", [("ad_leg_per", 1e-5), ("ad16_leg_per", 1e-5)])
def test_near_field_densities_are_independent(trees, name, delta):
    t = trees[name]
    nd = 3
    rng = np.random.default_rng(11)
    f = np.stack([t.fvals, -0.5 * t.fvals, rng.standard_normal(t.fvals.shape)], axis=2)
    f[t.nchild() > 0] = 0.0
    p3, _ = run(t, delta, 1e-6, hb.BFGT_PREC_SPLIT, f=f, nd=nd)
    p3 = p3.reshape(t.nboxes, t.npbox, nd)
    for d in range(nd):
        p1, _ = run(t, delta, 1e-6, hb.BFGT_PREC_SPLIT, f=np.ascontiguousarray(f[:, :, d]))
        np.testing.assert_array_equal(p3[:, :, d], p1.reshape(t.nboxes, t.npbox))


def test_fixed_point_plans_keep_the_fp64_near_field(trees):
    """eps < 1e-7: the FP64 near-field kernel (within 10 eps of the oracle)."""
    t = trees["ad_leg_per"]
    lv = t.leaves()
    p, _ = run(t, 1e-5, 1e-9, hb.BFGT_PREC_SPLIT)
    q, _ = run(t, 1e-5, 1e-9, hb.BFGT_PREC_FP64)
    ref = oracle.boxfgt(t, t.fvals, 1e-5, 1e-9).reshape(t.nboxes, -1)[lv]
    assert rel_l2(p.reshape(t.nboxes, -1)[lv], ref) < 1e-8
    np.testing.assert_array_equal(p, q)  # regime C: only the near field, and it is the FP64 kernel


@pytest.mark.parametrize("name,delta", [("ad_leg_per", 1e-5), ("ad16_leg_per", 1e-5), ("uni3_leg_free", 1e-5)])
def test_gradient_and_hessian_near_field_on_tensor_cores(trees, name, delta):
    """ifpgh = 3 in regime C: the derivative tables (tabx_loc, tabxx_loc) through
    the same tensor-core kernel, within min(2e-6, 20 eps) of the oracle's
    g2d_tens_prod_to_pghloc restatement."""
    import torch
    t = trees[name]
    lv = t.leaves()
    eps = 1e-6
    plan = hb.Plan(t, delta, eps, precision=hb.BFGT_PREC_SPLIT)
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    p = torch.zeros_like(f)
    g = torch.zeros(2 * f.numel(), dtype=torch.float64, device="cuda")
    h = torch.zeros(3 * f.numel(), dtype=torch.float64, device="cuda")
    plan.execute_pgh(3, f, p, g, h)
    plan.check()
    plan.close()
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 3)
    leaf = lambda v: v.reshape(t.nboxes, -1)[lv]  # noqa: E731
    assert rel_l2(leaf(p.cpu().numpy()), leaf(rp)) < 1e-6
    assert rel_l2(leaf(g.cpu().numpy()), leaf(rg)) < 2e-6
    assert rel_l2(leaf(h.cpu().numpy()), leaf(rh)) < 2e-6
