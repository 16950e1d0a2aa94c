"""The product's host-side step-0 precomputation (tables, band patterns and
interaction lists of bfgt/boxfgt.f:472-703) against the oracle's, bit for bit.
Runs without a GPU."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

from test_oracle import CASES


@pytest.mark.parametrize("name,delta,eps", CASES + [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9)])
def test_lists_and_tables_bit_exact(trees, name, delta, eps):
    t = trees[name]
    d, o = hb.host_plan_dump(t, delta, eps)
    _, info, it = oracle.boxfgt(t, t.fvals, delta, eps, with_info=True)
    assert d["npwlevel"] == info.npwlevel
    assert d["npw"] == info.npw
    assert d["regime"] == info.regime
    assert d["nlevstart"] == info.nlevstart
    assert d["nlevend"] == info.nlevend
    assert d["mnlist1"] == info.mnlist1
    assert d["nleafbox"] == info.nleafbox
    assert d["iperiod_int"] == info.iperiod_int
    # itree colleague arrays recomputed as bfgtmain does (boxfgt.f:516-528)
    np.testing.assert_array_equal(o["itree"], it)
    np.testing.assert_array_equal(o["ifpwexp"], info.ifpwexp)
    np.testing.assert_array_equal(o["nlist1"], info.nlist1)
    for b in range(t.nboxes):
        np.testing.assert_array_equal(o["list1"][b, : o["nlist1"][b]], info.list1[b, : info.nlist1[b]])
        np.testing.assert_array_equal(o["listpw"][b, : o["nlistpw"][b]], info.listpw[b, : info.nlistpw[b]])
    np.testing.assert_array_equal(o["nlistpw"], info.nlistpw)
    # near-field band patterns and tables
    np.testing.assert_array_equal(o["ind_loc"], info.ind_loc)
    np.testing.assert_array_equal(o["tab_loc"], info.tab_loc)
    np.testing.assert_array_equal(o["ts"], info.ts)
    np.testing.assert_array_equal(o["ws"], info.ws)


def test_config1_plan_scalars():
    """Uniform level-5 tree, Legendre order 8, delta=1e-3, eps=1e-9: npwlevel 2, npw 60, PW only."""
    g = np.array([[0.1, 0.2, 0.07, 0.5]])
    t = hb.build_uniform(5, g, norder=8, ipoly=0, iperiod=1)
    d, _ = hb.host_plan_dump(t, 1e-3, 1e-9)
    assert (d["npwlevel"], d["npw"], d["regime"], d["nnear_targets"], d["npwleaves"]) == (2, 60, 1, 0, 1024)


def test_invalid_tree_is_rejected():
    g = np.array([[0.1, 0.2, 0.07, 0.5]])
    t = hb.build_uniform(2, g, norder=8)
    bad = t.copy()
    bad.itree[bad.iptr[3] - 1] = 3          # nchild(1) = 3
    with pytest.raises(hb.BfgtError):
        hb.host_plan_dump(bad, 1e-3, 1e-9)
    bad = t.copy()
    bad.iptr[2] += 1                         # iptr inconsistent with nboxes
    with pytest.raises(hb.BfgtError):
        hb.host_plan_dump(bad, 1e-3, 1e-9)
    with pytest.raises(hb.BfgtError):
        hb.host_plan_dump(t, -1.0, 1e-9)     # delta <= 0


def test_npw_beyond_reference_capacity_is_rejected():
    """The reference sizes ws(200), ts(200) (boxfgt.f:434) without a check; here a
    transform that would need more than 200 plane waves is rejected."""
    g = hb.gauss_params(np.array([[0.1, 0.2]]), np.array([0.2]), np.array([1.0]))
    t = hb.build_uniform(0, g, norder=8, ipoly=0, iperiod=1)
    with pytest.raises(hb.BfgtError, match="npw > 200"):
        hb.host_plan_dump(t, 1e-5, 1e-9)
