"""Batches of plans (bfgt_batch_*): independent trees with their own delta,
eps, order, nd and precision, run with one launch per stage and kernel
variant over packed leaf arrays.

Each plan's slice of a batched execute must equal, bit for bit, the same
plan executed alone (the batched kernels do the same arithmetic in the same
order), and match the oracle to the precision's bar: FP64 within 1e-11
relative L2, split precision within 1e-6 (and 10*eps).  A scaled-down form of
the uneven-trees configuration (order 8, nd = 8, delta log-uniform in
[1e-5, 1e-1] so that all three regimes occur) is checked against the oracle.
"""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

from conftest import gauss_sum

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def leaf_values(t, nd, seed):
    """fvals(nd, npbox, nboxes) as (nboxes, npbox, nd): the tree's density
    scaled per density, one density replaced by noise (leaf boxes only)."""
    rng = np.random.default_rng(seed)
    f = np.repeat(t.fvals[:, :, None], nd, axis=2) * rng.uniform(0.5, 2.0, nd)[None, None, :]
    if nd > 1:
        f[:, :, nd - 1] = rng.standard_normal(f[:, :, nd - 1].shape)
    f[t.nchild() > 0] = 0.0
    return np.ascontiguousarray(f)


def run_batch(specs, graph=False):
    """specs: list of (tree, delta, eps, nd, precision).  Returns the batched
    results per plan, the single-plan results and the batch info."""
    import torch
    plans = [hb.Plan(t, d, e, nd=nd, precision=p) for (t, d, e, nd, p) in specs]
    batch = hb.Batch(plans)
    off = batch.offsets
    fv = [leaf_values(t, nd, 100 + i) for i, (t, _, _, nd, _) in enumerate(specs)]
    F = torch.from_numpy(np.concatenate([f.reshape(-1) for f in fv])).cuda()
    assert F.numel() == off[-1]
    P = torch.zeros_like(F)
    if graph:
        batch.graph_capture(F, P)
        batch.graph_launch()
    else:
        batch.execute(F, P)
    batch.check()
    got = P.cpu().numpy()
    info = batch.info()
    singles = []
    for i, pl in enumerate(plans):
        f = torch.from_numpy(fv[i].reshape(-1)).cuda()
        p = torch.zeros_like(f)
        pl.execute(f, p)
        pl.check()
        singles.append(p.cpu().numpy())
    out = [got[off[i]:off[i + 1]] for i in range(len(plans))]
    batch.close()
    for pl in plans:
        pl.close()
    return out, singles, fv, info


def check_oracle(specs, out, fv):
    for (t, d, e, nd, p), got, f in zip(specs, out, fv):
        ref = oracle.boxfgt(t, f, d, e, nd=nd).reshape(t.nboxes, -1)
        lv = t.leaves()
        err = rel_l2(got.reshape(t.nboxes, -1)[lv], ref[lv])
        bar = 1e-11 if p == hb.BFGT_PREC_FP64 else min(1e-6, 10 * e)
        assert err <= bar, (d, e, nd, p, err)


def test_batch_mixed_plans(trees):
    S, F = hb.BFGT_PREC_SPLIT, hb.BFGT_PREC_FP64
    specs = [(trees["ad16_leg_per"], 1e-4, 1e-6, 1, S),
             (trees["ad_leg_per"], 1e-4, 1e-6, 2, S),       # order 8, nd 2
             (trees["uni3_leg_per"], 1e-3, 1e-9, 1, S),
             (trees["ad_cheb_free"], 1e-4, 1e-9, 1, F),     # an FP64 plan in the batch
             (trees["uni3_leg_per"], 4e-4, 1e-9, 1, S),     # near field only
             (trees["uni3_cheb_per"], 1e-2, 1e-6, 3, S),    # periodic Fourier regime
             (trees["ad16_leg_per"], 1e-2, 1e-6, 1, S),     # odd npw
             (trees["lev1_leaf_per"], 1e-3, 1e-6, 1, F),
             (trees["ad_leg_per"], 1e-3, 1e-10, 3, S),      # fixed-point slices, 5 digits, packed
             (trees["ad16_leg_per"], 1e-3, 1e-8, 1, S)]     # fixed-point slices, 4 digits
    out, singles, fv, info = run_batch(specs)
    for a, b in zip(out, singles):
        np.testing.assert_array_equal(a, b)
    check_oracle(specs, out, fv)
    assert info["plans"] == len(specs)


def test_batch_graph_replay_matches(trees):
    S = hb.BFGT_PREC_SPLIT
    specs = [(trees["ad16_leg_per"], 1e-4, 1e-6, 1, S), (trees["ad_leg_per"], 1e-3, 1e-6, 1, S),
             (trees["ad_cheb_free"], 1e-4, 1e-6, 2, S)]
    out, singles, _, _ = run_batch(specs, graph=True)
    for a, b in zip(out, singles):
        np.testing.assert_array_equal(a, b)


def uneven_trees(ntrees, seed, lo=200, hi=3000):
    """Scaled-down uneven-trees configuration: order-8 periodic trees grown
    until their leaf count is log-uniform in [lo, hi], each a sum of 5-30
    Gaussians (widths log-uniform in [2e-3, 5e-2]), delta log-uniform in
    [1e-5, 1e-1], eps 1e-6, nd 8."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ntrees):
        ng = int(rng.integers(5, 31))
        g = gauss_sum(1000 + i, ng, 2e-3, 5e-2, amp="normal", log_width=True)
        target = np.exp(rng.uniform(np.log(lo), np.log(hi)))
        t = None
        for tail in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9):
            t = hb.build_adaptive(g, norder=8, ipoly=0, iperiod=1, eps=tail, maxlev=8)
            if len(t.leaves()) >= target:
                break
        delta = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-1))))
        out.append((t, delta, 1e-6, 8, hb.BFGT_PREC_SPLIT))
    return out


def test_batch_uneven_trees_nd8():
    specs = uneven_trees(8, 6)
    out, singles, fv, info = run_batch(specs)
    for a, b in zip(out, singles):
        np.testing.assert_array_equal(a, b)
    check_oracle(specs, out, fv)
    # one launch per stage and kernel variant, not per tree
    assert info["launches"] < 2 * len(specs)


def test_batch_adjoint_matches_single_plan_adjoints(trees):
    """bfgt_batch_execute_adjoint: each plan's slice equals its own
    bfgt_plan_execute_adjoint bit for bit, and sum(g K f) = sum(f K^T g)."""
    import torch
    S, F = hb.BFGT_PREC_SPLIT, hb.BFGT_PREC_FP64
    specs = [(trees["ad16_leg_per"], 1e-4, 1e-6, 1, S), (trees["ad_cheb_free"], 1e-4, 1e-9, 2, F),
             (trees["uni3_leg_per"], 4e-4, 1e-9, 1, S), (trees["lev1_leaf_per"], 1e-3, 1e-6, 1, S)]
    plans = [hb.Plan(t, d, e, nd=nd, precision=p) for (t, d, e, nd, p) in specs]
    batch = hb.Batch(plans)
    off = batch.offsets
    g = [leaf_values(t, nd, 300 + i) for i, (t, _, _, nd, _) in enumerate(specs)]
    f = [leaf_values(t, nd, 400 + i) for i, (t, _, _, nd, _) in enumerate(specs)]
    G = torch.from_numpy(np.concatenate([x.reshape(-1) for x in g])).cuda()
    Fv = torch.from_numpy(np.concatenate([x.reshape(-1) for x in f])).cuda()
    KtG = torch.zeros_like(G)
    KF = torch.zeros_like(Fv)
    batch.execute_adjoint(G, KtG)
    batch.execute(Fv, KF)
    batch.check()
    for i, pl in enumerate(plans):
        gi = torch.from_numpy(g[i].reshape(-1)).cuda()
        ai = torch.zeros_like(gi)
        pl.execute_adjoint(gi, ai)
        np.testing.assert_array_equal(KtG[off[i]:off[i + 1]].cpu().numpy(), ai.cpu().numpy())
    a, b = torch.dot(KF, G).item(), torch.dot(Fv, KtG).item()
    assert abs(a - b) <= 1e-6 * KF.norm().item() * G.norm().item()
    batch.close()
    for pl in plans:
        pl.close()


def test_batch_refuses_a_repeated_plan(trees):
    """A plan owns its expansion scratch and arrival counters, so one plan
    listed twice in a batch would mix two transforms' partial sums:
    bfgt_batch_create refuses it (BFGT_ERR_ARG) and creates nothing."""
    a = hb.Plan(trees["ad_leg_per"], 1e-4, 1e-6, precision=hb.BFGT_PREC_SPLIT)
    b = hb.Plan(trees["uni3_leg_per"], 1e-3, 1e-9)
    with pytest.raises(hb.BfgtError, match="repeats plan"):
        hb.Batch([a, b, a])
    batch = hb.Batch([a, b])  # the same plans once each are fine
    batch.close()
    a.close()
    b.close()
