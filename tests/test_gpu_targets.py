"""Extra targets (boxfgt.f step 11, ifpghtarg = 1..3) on the GPU against the
oracle's restatement (treedata_trans_nd + treedata_evalt_nd with
pts_tree_sort).  Values within 1e-12 relative L2: the same sums in the same
order.  Targets include points on box edges and corners, where the leaf
assignment (child 1 + (x >= cx) + 2 (y >= cy)) decides which interpolant is
used; a wrong assignment shows up far above the bar."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def targets(t, seed, n=4000):
    rng = np.random.default_rng(seed)
    h = t.boxsize[t.nlevels]
    edge = np.arange(-6, 7) * h
    edge = edge[np.abs(edge) < 0.5]   # inside the box: no polynomial extrapolation
    grid = np.stack(np.meshgrid(edge, edge), -1).reshape(-1, 2)
    corners = np.array([[-0.5, -0.5], [0.0, 0.0], [0.25, -0.25], [0.5 - 1e-12, 0.5 - 1e-12]])
    return np.ascontiguousarray(np.concatenate([rng.uniform(-0.5, 0.5, (n, 2)), grid, corners]))


@pytest.mark.parametrize("name,delta,eps,ifpgh,ifpghtarg",
                         [("ad_leg_per", 1e-4, 1e-6, 1, 1), ("ad_cheb_free", 1e-4, 1e-9, 3, 3),
                          ("ad_leg_per", 1e-3, 1e-9, 1, 3), ("uni3_leg_per", 1e-3, 1e-9, 2, 2),
                          ("ad16_leg_per", 1e-4, 1e-6, 1, 2)])
def test_boxfgt_targets_match_oracle(trees, name, delta, eps, ifpgh, ifpghtarg):
    t = trees[name]
    tg = targets(t, 1)
    nt = len(tg)
    m = t.nboxes * t.npbox
    pot = np.zeros(m)
    grad = np.zeros(2 * m) if ifpgh >= 2 else None
    hess = np.zeros(3 * m) if ifpgh == 3 else None
    pote, grade, hesse = np.zeros(nt), np.zeros(2 * nt), np.zeros(3 * nt)
    ti = np.zeros(20)
    hb.boxfgt(1, 2, delta, eps, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree, t.itree.copy(),
              t.iptr, t.centers, t.boxsize, np.ascontiguousarray(t.fvals), ifpgh, pot, grad, hess, 0, nt,
              tg.reshape(-1), ifpghtarg, pote, grade, hesse, ti)
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, delta, eps, max(ifpgh, ifpghtarg))
    ep, _ = oracle.eval_targets(t, rp, tg)
    assert rel_l2(pote, ep[:, 0]) < 1e-12
    if ifpghtarg >= 2:
        eg, _ = oracle.eval_targets(t, rg, tg, nd=2)
        assert rel_l2(grade, eg.reshape(-1)) < 1e-12
    if ifpghtarg == 3:
        eh, _ = oracle.eval_targets(t, rh, tg, nd=3)
        assert rel_l2(hesse, eh.reshape(-1)) < 1e-12


def test_eval_targets_device_entry_nd2(trees):
    import torch
    t = trees["ad_cheb_free"]
    nd = 2
    rng = np.random.default_rng(2)
    vals = rng.standard_normal((t.nboxes, t.npbox, nd))
    tg = targets(t, 3, 1000)
    plan = hb.Plan(t, 1e-4, 1e-6, nd=nd)
    dv = torch.from_numpy(vals.reshape(-1)).cuda()
    dt = torch.from_numpy(tg.reshape(-1)).cuda()
    out = torch.zeros(nd * len(tg), dtype=torch.float64, device="cuda")
    plan.eval_targets(1, dv, len(tg), dt, out)
    plan.eval_targets(1, dv, 0, dt, out)   # no targets: nothing to do
    torch.cuda.synchronize()
    plan.close()
    ref, _ = oracle.eval_targets(t, vals, tg, nd=nd)
    assert rel_l2(out.cpu().numpy(), ref.reshape(-1)) < 1e-12
