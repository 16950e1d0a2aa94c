"""The interaction lists of the product's step-0 precomputation against their
geometric meaning, derived here from box positions alone (no code shared with
the product or the oracle, which both restate the reference's list routines
step by step).  The definitions, from the comments and tests of
common/tree_routs_nd.f:

* colleagues of a box (computecoll, 106-250): the boxes of its level that it
  touches or is, in the periodic nearest image when the internal iperiod is 1;
* plane-wave flags (gnd_find_pwexp_boxes, 1266-1325): every box below the
  cutoff level; at the cutoff level a non-leaf box, or a leaf with a non-leaf
  colleague; the root when the cutoff level is 0 or less; none when the
  cutoff level is below the tree;
* list1 of a leaf at levels 1 .. nlevend (gnd_compute_modified_list1,
  864-1050): the leaves it touches at its own level (itself only without a
  plane-wave expansion), one level coarser, and one level finer when its
  level is above the cutoff level; the root's list is itself when the root is
  a leaf;
* listpw of a box at the cutoff level (gnd_compute_listpw, 1564-1615): its
  colleagues other than itself when either of the two has children.

Lists are compared as sets (their order is the reference's enumeration order,
checked bit for bit against the oracle elsewhere).  Runs without a GPU."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb

from test_oracle import CASES


def geometry(t, iper):
    lev = t.ilevel().astype(int)
    bs = t.boxsize[lev]
    cen = t.centers
    L0 = t.boxsize[0]

    def dist(a, b):
        d = np.abs(cen[a] - cen[b])
        if iper:
            d = np.minimum(d, L0 - d)
        return d

    # two boxes touch (or coincide) when, in both coordinates, their centres
    # are at most half the sum of their sizes apart; boxes that do not touch
    # are at least half the smaller size further apart
    def touch(a, b):
        lim = (bs[a] + bs[b]) / 2 + 0.25 * np.minimum(bs[a], bs[b])
        return np.all(dist(a, b) <= lim[:, None] if np.ndim(lim) else dist(a, b) <= lim, axis=-1)

    return lev, touch


def geometric_lists(t, d):
    nb = t.nboxes
    nch = t.nchild()
    npwlevel, nlevels, iper = d["npwlevel"], t.nlevels, d["iperiod_int"]
    lev, touch = geometry(t, iper)
    boxes = np.arange(nb)
    coll = [set() for _ in range(nb)]
    for l in range(nlevels + 1):
        at = boxes[lev == l]
        for b in at:
            coll[b] = set(at[touch(np.full(len(at), b), at)].tolist())
    ncut = max(npwlevel, 0)
    ifpw = np.zeros(nb, int)
    if npwlevel <= nlevels:
        ifpw[lev > ncut] = 1
        for b in boxes[lev == ncut]:
            if nch[b] > 0 or any(nch[j] > 0 for j in coll[b]):
                ifpw[b] = 1
        if npwlevel <= 0:
            ifpw[0] = 1
    nlevend = nlevels if npwlevel >= nlevels else npwlevel
    leaves = boxes[nch == 0]
    list1 = [set() for _ in range(nb)]
    if nch[0] == 0:
        list1[0] = {0}
    for b in leaves:
        lb = lev[b]
        if lb < 1 or lb > nlevend:
            continue
        cand = leaves[np.abs(lev[leaves] - lb) <= 1]
        cand = cand[touch(np.full(len(cand), b), cand)]
        s = set()
        for c in cand.tolist():
            if lev[c] == lb + 1 and not lb < npwlevel:
                continue
            if c == b and ifpw[b] == 1:
                continue
            s.add(c)
        list1[b] = s
    listpw = [set() for _ in range(nb)]
    if npwlevel <= nlevels:
        for b in boxes[lev == ncut]:
            listpw[b] = {j for j in coll[b] if j != b and (nch[j] > 0 or nch[b] > 0)}
    return coll, ifpw, list1, listpw


# (deltas of 1e-4 and below put most leaves of the adaptive trees in the near
# field, with list1 entries one level coarser and finer)
@pytest.mark.parametrize("name,delta,eps", CASES + [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9),
                                                    ("lev1_leaf_per", 1e-3, 1e-6), ("ad_cheb_free", 1e-2, 1e-6),
                                                    ("ad_leg_per", 1e-5, 1e-6), ("ad_cheb_free", 3e-5, 1e-9),
                                                    ("ad16_leg_per", 3e-5, 1e-6)])
def test_lists_match_their_geometric_definition(trees, name, delta, eps):
    t = trees[name]
    d, o = hb.host_plan_dump(t, delta, eps)
    coll, ifpw, list1, listpw = geometric_lists(t, d)
    it = o["itree"]
    s6, s7 = t.iptr[5] - 1, t.iptr[6] - 1
    ncoll = it[s6:s6 + t.nboxes]
    colls = it[s7:s7 + 9 * t.nboxes].reshape(t.nboxes, 9)
    for b in range(t.nboxes):
        got = set((colls[b, :ncoll[b]] - 1).tolist())
        assert got == coll[b], ("colleagues", b)
    np.testing.assert_array_equal(o["ifpwexp"], ifpw)
    for b in range(t.nboxes):
        assert set((o["list1"][b, :o["nlist1"][b]] - 1).tolist()) == list1[b], ("list1", b)
        assert set((o["listpw"][b, :o["nlistpw"][b]] - 1).tolist()) == listpw[b], ("listpw", b)
