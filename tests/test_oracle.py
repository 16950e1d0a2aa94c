"""The oracle (C restatement of bfgt/boxfgt.f) against the independent FP64
quadrature and against the reference's own known-answer test
(hpots/test_initpot.f:58-80, 239-250, 346-380)."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle, quad


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def leaf_vals(tree, v):
    return np.asarray(v).reshape(tree.nboxes, -1)[tree.leaves()]


CASES = [
    ("uni3_leg_per", 1e-3, 1e-9),    # PW + cutoff translation (regime B)
    ("uni3_cheb_per", 1e-2, 1e-6),   # periodic Fourier regime (A)
    ("uni3_leg_per", 4e-4, 1e-9),    # near field only (C)
    ("uni3_leg_free", 1e-3, 1e-9),
    ("uni3_leg_free", 1e-1, 1e-6),   # free space, cutoff at the root
    ("ad_leg_per", 1e-4, 1e-6),      # adaptive: PW below the cutoff + near field above
    ("ad_cheb_free", 1e-4, 1e-9),
    ("ad_leg_per", 1e-2, 1e-9),
    ("lev1_leaf_per", 1e-3, 1e-6),   # periodic level-1 images in the near field
    ("lev1_leaf_per", 2e-2, 1e-9),
]


@pytest.mark.parametrize("name,delta,eps", CASES)
def test_oracle_vs_quadrature(trees, name, delta, eps):
    t = trees[name]
    if t.nboxes > 1500:
        pytest.skip("tree too large for the quadrature oracle")
    p = oracle.boxfgt(t, t.fvals, delta, eps)
    q = quad.direct_pot(t, t.fvals, delta)
    err = rel_l2(leaf_vals(t, p), leaf_vals(t, q))
    assert err < 10 * eps, err


def kat_tree(level, ipoly, n=8):
    """Uniform periodic tree with f = sin(2 pi s1 x) cos(2 pi s2 y), s1 = s2 = 2 (test_initpot.f:319)."""
    g = hb.gauss_params(np.zeros((1, 2)), np.ones(1), np.zeros(1))
    t = hb.build_uniform(level, g, norder=n, ipoly=ipoly, iperiod=1)
    xy = t.grid_points()
    t.fvals = np.sin(2 * 2 * np.pi * xy[..., 0]) * np.cos(2 * 2 * np.pi * xy[..., 1])
    return t


@pytest.mark.parametrize("delta,level,regime", [
    (4e-5, 5, 2),    # test_initpot.f: dt = 1e-5, delta = 4 dt, eps = 1e-9 (near field only)
    (4e-5, 6, 1),    # same transform with the cutoff above the leaves (PW)
    (1e-3, 4, 1),
    (1e-2, 4, 0),    # periodic Fourier regime
])
def test_oracle_fourier_kat(delta, level, regime):
    """pot / (pi delta) = exp(-pi^2 (s1^2+s2^2) delta) f  (hpots/test_initpot.f:367-373)."""
    eps = 1e-9
    t = kat_tree(level, ipoly=1)
    p, info, _ = oracle.boxfgt(t, t.fvals, delta, eps, with_info=True)
    assert info.regime == regime
    lv = t.leaves()
    exact = np.exp(-np.pi ** 2 * 8 * delta) * t.fvals[lv]
    got = p.reshape(t.nboxes, -1)[lv] / (np.pi * delta)
    err = np.abs(got - exact).max() / np.abs(exact).max()
    assert err < 1e-7, err   # interpolation error of the n=8 leaf grid dominates


def test_oracle_golden_vectors():
    """Committed fixtures (tests/golden/make_golden.py): analytic KAT values and quadrature values."""
    import json
    from pathlib import Path
    g = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())
    for case in g["cases"]:
        gauss = np.array(case["gauss"])
        if case["kind"] == "uniform":
            t = hb.build_uniform(case["level"], gauss, norder=case["norder"], ipoly=case["ipoly"],
                                 iperiod=case["iperiod"])
        else:
            t = hb.build_adaptive(gauss, norder=case["norder"], ipoly=case["ipoly"], iperiod=case["iperiod"],
                                  eps=case["tree_eps"], maxlev=case["maxlev"])
        if case.get("density") == "fourier22":
            xy = t.grid_points()
            t.fvals = np.sin(4 * np.pi * xy[..., 0]) * np.cos(4 * np.pi * xy[..., 1])
        assert t.nboxes == case["nboxes"], "tree generator changed"
        p = oracle.boxfgt(t, t.fvals, case["delta"], case["eps"]).reshape(t.nboxes, -1)
        idx = np.array(case["sample_idx"])
        ref = np.array(case["sample_pot"])
        got = p[idx[:, 0], idx[:, 1]]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err < 10 * case["eps"], (case["name"], err)


PGH_CASES = [("uni3_leg_per", 1e-3, 1e-9), ("uni3_cheb_per", 1e-2, 1e-9), ("uni3_leg_per", 4e-4, 1e-9),
             ("uni3_leg_free", 1e-3, 1e-9), ("ad_leg_per", 1e-4, 1e-9), ("lev1_leaf_per", 1e-3, 1e-9)]


@pytest.mark.parametrize("name,delta,eps", PGH_CASES)
def test_oracle_gradient_hessian_vs_quadrature(trees, name, delta, eps):
    """ifpgh = 3 (g2d_pw2pgh, g2d_tens_prod_to_pghloc restated) against the
    direct quadrature of the kernel's first and second derivatives.  The
    derivatives carry the transform's error times 1/sqrt(delta) per order, so
    the bars are 100 eps (gradient) and 1000 eps (hessian); pot must equal the
    ifpgh = 1 result bit for bit."""
    t = trees[name]
    p1 = oracle.boxfgt(t, t.fvals, delta, eps)
    p, g, h = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 3)
    np.testing.assert_array_equal(p, p1)
    qp, qg, qh = quad.direct_pgh(t, t.fvals, delta, ifpgh=3)
    assert rel_l2(leaf_vals(t, p), leaf_vals(t, qp)) < 10 * eps
    assert rel_l2(leaf_vals(t, g), leaf_vals(t, qg)) < 100 * eps
    assert rel_l2(leaf_vals(t, h), leaf_vals(t, qh)) < 1000 * eps
    p2, g2, h2 = oracle.boxfgt_pgh(t, t.fvals, delta, eps, 2)
    np.testing.assert_array_equal(p2, p1)
    np.testing.assert_array_equal(g2, g)
    assert h2 is None


def test_oracle_gradient_multiple_densities(trees):
    t = trees["ad_cheb_free"]
    nd = 2
    rng = np.random.default_rng(3)
    fv = np.stack([t.fvals, rng.standard_normal(t.fvals.shape) * (t.nchild() == 0)[:, None]], axis=2)
    _, g, _ = oracle.boxfgt_pgh(t, fv, 1e-3, 1e-9, 2, nd=nd)
    _, qg, _ = quad.direct_pgh(t, fv, 1e-3, nd=nd, ifpgh=2)
    assert rel_l2(leaf_vals(t, g), leaf_vals(t, qg)) < 1e-7


def test_oracle_targets_interpolate_and_sort(trees):
    """Step 11 restated (treedata_evalt_nd with pts_tree_sort): every target
    lands in the leaf that contains it, with points on an edge going to the
    upper child (find_childbox_ind's dx >= 0), and interpolating the density's
    own leaf values reproduces it to the tree's resolution."""
    from fgt_autograd import gauss_at_points
    t = trees["ad_leg_per"]
    rng = np.random.default_rng(0)
    h = t.boxsize[t.nlevels]
    edge = (np.arange(-4, 5) * h)
    tg = np.concatenate([rng.uniform(-0.5, 0.5, (3000, 2)), np.stack(np.meshgrid(edge, edge), -1).reshape(-1, 2)])
    out, leaf = oracle.eval_targets(t, t.fvals, tg)
    lev = t.ilevel()[leaf - 1]
    c = t.centers[leaf - 1]
    half = t.boxsize[lev][:, None] / 2
    assert np.all(t.nchild()[leaf - 1] == 0)
    assert np.all((tg >= c - half) & (tg < c + half))
    from conftest import gauss_sum
    g6 = gauss_sum(2, 6, 0.01, 0.05, amp="normal", log_width=True)
    assert np.abs(out[:, 0] - gauss_at_points(tg, g6)).max() < 1e-5
