"""Caller-side tree generator: valid reference layout, 2:1 balance, colleagues."""
import numpy as np
import pytest


def check_tree(t):
    nb, nl = t.nboxes, t.nlevels
    lad = t.laddr()
    assert lad[0, 0] == 1 and lad[0, 1] == 1
    for l in range(1, nl + 1):
        assert lad[l, 0] == lad[l - 1, 1] + 1
    lev, par, nch, ich = t.ilevel(), t.iparent(), t.nchild(), t.ichild()
    for l in range(nl + 1):
        assert (lev[lad[l, 0] - 1: lad[l, 1]] == l).all()
    for b in range(nb):
        if nch[b]:
            assert nch[b] == 4
            for j in range(4):
                c = ich[b, j] - 1
                assert par[c] == b + 1
                # child order mm, pm, mp, pp (common/pts_tree_nd.f:1418-1460)
                sx = -1 if j in (0, 2) else 1
                sy = -1 if j in (0, 1) else 1
                h = t.boxsize[lev[c]] / 2
                assert np.allclose(t.centers[c], t.centers[b] + np.array([sx, sy]) * h)


def leaf_touch_levels(t):
    """max level difference between touching leaves (periodic aware)."""
    lv = t.leaves()
    lev = t.ilevel()[lv]
    c = t.centers[lv]
    hs = t.boxsize[lev] / 2
    L = t.boxsize[0]
    worst = 0
    for i in range(len(lv)):
        d = np.abs(c - c[i])
        if t.iperiod:
            d = np.minimum(d, L - d)
        touch = np.all(d <= (hs + hs[i])[:, None] * (1 + 1e-9), axis=1)
        worst = max(worst, int(np.abs(lev[touch] - lev[i]).max()))
    return worst


@pytest.mark.parametrize("name", ["ad_leg_per", "ad_cheb_free", "lev1_leaf_per", "uni3_leg_per"])
def test_tree_layout_and_balance(trees, name):
    t = trees[name]
    check_tree(t)
    assert leaf_touch_levels(t) <= 1


def test_colleagues(trees):
    t = trees["ad_leg_per"]
    nc, co = t.ncoll(), t.coll()
    lev = t.ilevel()
    L = t.boxsize[0]
    for b in range(t.nboxes):
        cs = co[b, : nc[b]] - 1
        assert (lev[cs] == lev[b]).all()
        d = np.abs(t.centers[cs] - t.centers[b])
        d = np.minimum(d, L - d)
        assert (d <= 1.05 * t.boxsize[lev[b]]).all()
        assert b in cs
