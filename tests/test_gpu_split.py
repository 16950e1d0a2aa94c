"""Split-precision tensor-core path (tcgen05, BF16 slices) vs the FP64 oracle.

Specified bar: relative L2 error over leaf values <= min(1e-6, 10*eps)
against the FP64 oracle.  eps >= 1e-7 runs three floating slices (about
1e-6); smaller eps runs fixed-point (Ozaki) slices, 4 of them down to
eps = 1e-9 and 5 down to 1e-11; below that a split plan is refused."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

from conftest import gauss_sum

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-6


def split_bar(eps):
    return min(SPLIT_TOL, 10 * eps)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run_split(t, delta, eps, fvals=None, nd=1, pot0=None):
    import torch
    plan = hb.Plan(t, delta, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT)
    fv = t.fvals if fvals is None else fvals
    f = torch.from_numpy(np.ascontiguousarray(fv).reshape(-1)).cuda()
    p = torch.zeros_like(f) if pot0 is None else torch.from_numpy(pot0.copy()).cuda()
    plan.execute(f, p)
    plan.check()
    out = p.cpu().numpy()
    info = plan.info()
    plan.close()
    return out, info


CASES = [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9), ("ad16_leg_per", 1e-2, 1e-6),
         ("ad_leg_per", 1e-4, 1e-6), ("ad_cheb_free", 1e-4, 1e-9), ("uni3_leg_per", 1e-3, 1e-9),
         ("uni3_cheb_per", 1e-2, 1e-6),
         # fixed-point slices: 4 digits (eps 1e-8, 1e-9), 5 digits (1e-10, 1e-11)
         ("ad16_leg_per", 1e-4, 1e-8), ("ad16_leg_per", 1e-2, 1e-9), ("ad_leg_per", 1e-4, 1e-10),
         ("ad16_leg_per", 1e-4, 1e-11), ("ad16_leg_per", 1e-2, 1e-11), ("uni3_cheb_per", 1e-2, 1e-10), ("lev1_leaf_per", 1e-3, 1e-9)]


@pytest.mark.parametrize("name,delta,eps", CASES)
def test_split_matches_oracle(trees, name, delta, eps):
    t = trees[name]
    got, info = run_split(t, delta, eps)
    ref = oracle.boxfgt(t, t.fvals, delta, eps)
    lv = t.leaves()
    err = rel_l2(got.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv])
    assert err < split_bar(eps), (err, info)


def test_split_refuses_eps_it_cannot_reach(trees):
    """Below eps = 1e-11 the fixed-point slices cannot promise 10*eps: plan
    creation fails with BFGT_ERR_CAPACITY and names the FP64 mode."""
    with pytest.raises(hb.BfgtError) as e:
        hb.Plan(trees["ad16_leg_per"], 1e-4, 1e-12, precision=hb.BFGT_PREC_SPLIT)
    assert e.value.code == 3
    assert "FP64" in str(e.value)


def test_split_benchmark_statistics_tree():
    """Adaptive order-16 tree with the benchmark's density statistics (smaller base level)."""
    rng = np.random.default_rng(2)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (20, 2)), np.exp(rng.uniform(np.log(1e-3), np.log(1e-2), 20)),
                        rng.standard_normal(20))
    t = hb.build_adaptive(g, norder=16, ipoly=0, iperiod=1, eps=1e-10, eta=1.0, minlev=6, maxlev=12)
    for delta, eps in [(1e-4, 1e-6), (1e-2, 1e-6), (1e-4, 1e-9), (1e-2, 1e-9)]:
        got, info = run_split(t, delta, eps)
        ref = oracle.boxfgt(t, t.fvals, delta, eps)
        lv = t.leaves()
        err = rel_l2(got.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv])
        assert err < split_bar(eps), (delta, eps, err, info)


@pytest.mark.parametrize("name,eps,nd", [("ad16_leg_per", 1e-6, 2), ("ad16_leg_per", 1e-9, 2),
                                         ("ad_leg_per", 1e-9, 5)])
def test_split_multiple_densities_and_accumulate(trees, name, eps, nd):
    t = trees[name]
    rng = np.random.default_rng(3)
    fv = np.stack([t.fvals] + [rng.standard_normal(t.fvals.shape) for _ in range(nd - 1)], axis=2)
    fv[t.nchild() > 0] = 0.0
    fv = np.ascontiguousarray(fv)
    pot0 = rng.standard_normal(t.nboxes * t.npbox * nd)
    got, _ = run_split(t, 1e-4, eps, fvals=fv, nd=nd, pot0=pot0)
    ref = oracle.boxfgt(t, fv, 1e-4, eps, nd=nd)
    lv = t.leaves()
    g = (got - pot0).reshape(t.nboxes, -1)[lv]
    assert rel_l2(g, ref.reshape(t.nboxes, -1)[lv]) < split_bar(eps)
    nonleaf = np.nonzero(t.nchild() > 0)[0]
    np.testing.assert_array_equal(got.reshape(t.nboxes, -1)[nonleaf], pot0.reshape(t.nboxes, -1)[nonleaf])


@pytest.mark.parametrize("eps", [1e-6, 1e-9])
def test_split_deterministic(trees, eps):
    t = trees["ad16_leg_per"]
    a, _ = run_split(t, 1e-4, eps)
    b, _ = run_split(t, 1e-4, eps)
    np.testing.assert_array_equal(a, b)


def test_bounded_wait_expiry_reports_timeout_and_context_survives(trees):
    """A wait limit of 0 makes every tensor-core pipeline wait give up at once:
    the kernels stop issuing, drain, free tensor memory and return; check()
    reports BFGT_ERR_TIMEOUT.  The next execute with the default limit on the
    same plan and context is correct."""
    import torch
    t = trees["ad16_leg_per"]
    delta, eps = 1e-4, 1e-6
    plan = hb.Plan(t, delta, eps, precision=hb.BFGT_PREC_SPLIT)
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    p = torch.zeros_like(f)
    plan.set_wait_limit(0)
    plan.execute(f, p)
    with pytest.raises(hb.BfgtError) as e:
        plan.check()
    assert e.value.code == 7
    plan.set_wait_limit(None)
    p.zero_()
    plan.execute(f, p)
    plan.check()
    got = p.cpu().numpy()
    plan.close()
    ref = oracle.boxfgt(t, t.fvals, delta, eps)
    lv = t.leaves()
    assert rel_l2(got.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv]) < SPLIT_TOL
