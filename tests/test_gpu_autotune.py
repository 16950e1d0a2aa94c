"""The tile-shape autotuner (bfgt_plan_autotune): it times the compiled FP64
tile shapes on the plan's own work lists, keeps the fastest, and later plans
of the same (norder, npw, nd) start with it.  Results must not change beyond
FP64 rounding (every shape computes the same sums, 1e-11 against the oracle),
the caller's arrays are untouched, and split plans have nothing to tune."""
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


def test_autotune_split_plan_is_a_no_op(trees):
    t = trees["ad16_leg_per"]
    plan = hb.Plan(t, 1e-4, 1e-6, precision=hb.BFGT_PREC_SPLIT)
    assert plan.autotune() == (0.0, 0.0, 0)
    assert plan.info()["form_tile"] == 0
    plan.close()
