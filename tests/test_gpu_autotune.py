"""The shape autotuner (bfgt_plan_autotune): it times the compiled FP64 tile
shapes on the plan's own work lists, keeps the fastest, and later plans of the
same (norder, npw, nd) start with it.  Results must not change beyond FP64
rounding (every shape computes the same sums, 1e-11 against the oracle), and
the caller's arrays are untouched.  Split plans: the form kernel's Y staging
and x tiles and the eval kernel's step groups and work (chunks or their column
halves) are timed; every choice gives the same bits as the untuned plan."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name,delta,eps", [("ad16_leg_per", 1e-4, 1e-6), ("ad_leg_per", 1e-3, 1e-9)])
def test_autotune_keeps_results_and_caches(trees, name, delta, eps):
    import torch
    t = trees[name]
    plan = hb.Plan(t, delta, eps)
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    p = torch.zeros_like(f)
    tf, te, ncand = plan.autotune()
    assert tf > 0 and te > 0 and ncand >= 2
    assert not p.any()                       # the caller's arrays are not used
    info = plan.info()
    plan.execute(f, p)
    plan.check()
    ref = oracle.boxfgt(t, t.fvals, delta, eps).reshape(t.nboxes, -1)
    lv = t.leaves()
    assert rel_l2(p.cpu().numpy().reshape(t.nboxes, -1)[lv], ref[lv]) < 1e-11
    again = hb.Plan(t, delta, eps)           # same shape: starts with the tuned tiles
    assert again.info()["form_tile"] == info["form_tile"]
    assert again.info()["eval_tile"] == info["eval_tile"]
    again.close()
    plan.close()


@pytest.mark.parametrize("name,delta,eps,nd", [("ad16_leg_per", 1e-4, 1e-6, 1), ("ad16_leg_per", 1e-3, 1e-9, 1),
                                               ("ad_leg_per", 1e-4, 1e-6, 3), ("uni3_leg_per", 1e-2, 1e-6, 1)])
def test_autotune_split_plan_same_bits(trees, name, delta, eps, nd):
    import torch
    t = trees[name]
    f0 = np.repeat(t.fvals[:, :, None], nd, axis=2) * np.linspace(1.0, 2.0, nd)[None, None, :]
    f = torch.from_numpy(np.ascontiguousarray(f0).reshape(-1)).cuda()
    base = hb.Plan(t, delta, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT)
    p0 = torch.zeros_like(f)
    base.execute(f, p0)
    base.check()
    plan = hb.Plan(t, delta, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT)
    tf, te, ncand = plan.autotune()
    assert tf > 0 and te > 0 and ncand >= 2
    p = torch.zeros_like(f)
    plan.execute(f, p)
    plan.check()
    np.testing.assert_array_equal(p.cpu().numpy(), p0.cpu().numpy())
    ref = oracle.boxfgt(t, t.fvals, delta, eps).reshape(t.nboxes, -1)
    lv = t.leaves()
    got = p.cpu().numpy().reshape(t.nboxes, t.npbox, nd)[lv, :, 0]
    assert rel_l2(got, ref[lv]) < min(1e-6, 10 * eps)
    # a batch made after tuning runs the tuned shapes: same bits again
    batch = hb.Batch([plan])
    pb = torch.zeros_like(f)
    batch.execute(f, pb)
    batch.check()
    np.testing.assert_array_equal(pb.cpu().numpy(), p0.cpu().numpy())
    batch.close()
    base.close()
    plan.close()


@pytest.mark.parametrize("name,delta,eps,nd", [("ad16_leg_per", 1e-4, 1e-6, 1), ("ad_leg_per", 1e-4, 1e-9, 1),
                                               ("ad_leg_per", 1e-4, 1e-6, 3)])
def test_eval_on_column_halves_same_bits(trees, monkeypatch, name, delta, eps, nd):
    """The eval kernel on the chunks' column halves (an autotuner choice, forced
    here through BFGT_SPLIT_EVAL_HALVES) gives the same bits, alone, in a batch
    and in the gradient and Hessian view: each output row's H and MMAs do not
    depend on the other rows."""
    import torch
    t = trees[name]
    f0 = np.repeat(t.fvals[:, :, None], nd, axis=2) * np.linspace(1.0, 2.0, nd)[None, None, :]
    f = torch.from_numpy(np.ascontiguousarray(f0).reshape(-1)).cuda()
    base = hb.Plan(t, delta, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT)
    p0 = torch.zeros_like(f)
    base.execute(f, p0)
    base.check()
    assert base.info()["split_shape"] < 1000
    monkeypatch.setenv("BFGT_SPLIT_EVAL_HALVES", "1")
    plan = hb.Plan(t, delta, eps, nd=nd, precision=hb.BFGT_PREC_SPLIT)
    assert plan.info()["split_shape"] >= 1000  # the halves are in use
    p = torch.zeros_like(f)
    plan.execute(f, p)
    plan.check()
    np.testing.assert_array_equal(p.cpu().numpy(), p0.cpu().numpy())
    batch = hb.Batch([plan])
    pb = torch.zeros_like(f)
    batch.execute(f, pb)
    batch.check()
    np.testing.assert_array_equal(pb.cpu().numpy(), p0.cpu().numpy())
    batch.close()
    # the gradient and Hessian view (3 nd densities, whole chunks or halves per CTA)
    outs = []
    for pl in (base, plan):
        pp = torch.zeros_like(f)
        g = torch.zeros(2 * f.numel(), dtype=torch.float64, device="cuda")
        h = torch.zeros(3 * f.numel(), dtype=torch.float64, device="cuda")
        pl.execute_pgh(3, f, pp, g, h)
        pl.check()
        outs.append([x.cpu().numpy() for x in (pp, g, h)])
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
    plan.close()
    base.close()
