"""The drop-in entry point boxfgt_ as a time-stepping solver uses it: the
same tree called again and again (hpots/hpots2dadap.f:103, 343) runs on a
cached plan, gives the same result as a fresh plan, and still rewrites the
colleague arrays of itree as the reference does (bfgt/boxfgt.f:516-528); the
precision selector puts boxfgt_ on the split path, with FP64 for calls split
precision cannot serve.  Bars: 1e-11 relative L2 against the oracle in FP64,
min(1e-6, 10 eps) in split precision."""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def call(t, delta, eps, itree=None, ifpgh=1):
    pot = np.zeros(t.npbox * t.nboxes)
    grad = np.zeros(2 * t.npbox * t.nboxes) if ifpgh >= 2 else None
    hess = np.zeros(3 * t.npbox * t.nboxes) if ifpgh >= 3 else None
    it = t.itree.copy() if itree is None else itree
    ti = np.zeros(20)
    hb.boxfgt(1, 2, delta, eps, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree, it, t.iptr,
              t.centers, t.boxsize, np.ascontiguousarray(t.fvals), ifpgh, pot, grad, hess, 0, 0, None, 0, None, None,
              None, ti)
    return pot, it, ti, grad, hess


@pytest.fixture(autouse=True)
def fresh_cache():
    hb.plan_cache_clear()
    hb.set_default_precision(hb.BFGT_PREC_FP64)
    yield
    hb.set_default_precision(hb.BFGT_PREC_FP64)
    hb.plan_cache_clear()


def test_repeated_calls_hit_the_cache_and_match(trees):
    t = trees["ad16_leg_per"]
    lv = t.leaves()
    p1, it1, ti1, _, _ = call(t, 1e-4, 1e-9)
    i1 = hb.plan_cache_info()
    # the caller's colleague arrays scrambled: a hit must rewrite them
    it = t.itree.copy()
    s = t.iptr[5] - 1
    it[s:] = -7
    p2, it2, ti2, _, _ = call(t, 1e-4, 1e-9, itree=it)
    i2 = hb.plan_cache_info()
    assert i2["hits"] == i1["hits"] + 1 and i2["entries"] == 1
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(it2, it1)
    assert ti2[0] < ti1[0]  # lookup instead of the step-0 precomputation
    ref, _, it_ref = oracle.boxfgt(t, t.fvals, 1e-4, 1e-9, with_info=True)
    np.testing.assert_array_equal(it2, it_ref)
    assert rel_l2(p2.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv]) < 1e-11


def test_changed_arguments_miss(trees):
    t = trees["ad_leg_per"]
    lv = t.leaves()
    call(t, 1e-4, 1e-6)
    m0 = hb.plan_cache_info()["misses"]
    p, _, _, _, _ = call(t, 2e-4, 1e-6)  # another delta: another plan
    assert hb.plan_cache_info()["misses"] == m0 + 1
    ref = oracle.boxfgt(t, t.fvals, 2e-4, 1e-6)
    assert rel_l2(p.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv]) < 1e-11
    # a moved box centre is another tree
    t2 = t.copy()
    t2.centers[0, -1] += 1e-3
    call(t2, 2e-4, 1e-6)
    assert hb.plan_cache_info()["misses"] == m0 + 2


def test_cache_off_gives_the_same_result(trees, monkeypatch):
    t = trees["ad16_leg_per"]
    a, _, _, _, _ = call(t, 1e-3, 1e-6)
    monkeypatch.setenv("BFGT_PLAN_CACHE", "0")
    hb.plan_cache_clear()
    b, _, _, _, _ = call(t, 1e-3, 1e-6)
    assert hb.plan_cache_info()["entries"] == 0
    np.testing.assert_array_equal(a, b)


def test_cached_plan_serves_gradient_and_hessian_calls(trees):
    t = trees["ad16_leg_per"]
    lv = t.leaves()
    call(t, 1e-4, 1e-9)
    p, _, _, g, h = call(t, 1e-4, 1e-9, ifpgh=3)
    assert hb.plan_cache_info()["hits"] >= 1
    rp, rg, rh = oracle.boxfgt_pgh(t, t.fvals, 1e-4, 1e-9, 3)
    leaf = lambda v, k: v.reshape(t.nboxes, -1)[lv]  # noqa: E731
    assert rel_l2(leaf(p, 1), leaf(rp, 1)) < 1e-11
    assert rel_l2(leaf(g, 2), leaf(rg, 2)) < 1e-11
    assert rel_l2(leaf(h, 3), leaf(rh, 3)) < 1e-11


@pytest.mark.parametrize("name,delta,eps", [("ad16_leg_per", 1e-4, 1e-6), ("ad16_leg_per", 1e-3, 1e-9),
                                            ("ad_cheb_free", 1e-4, 1e-6)])
def test_split_precision_through_boxfgt(trees, name, delta, eps):
    t = trees[name]
    lv = t.leaves()
    hb.set_default_precision(hb.BFGT_PREC_SPLIT)
    p, _, _, _, _ = call(t, delta, eps)
    p2, _, _, _, _ = call(t, delta, eps)  # cached split plan
    np.testing.assert_array_equal(p, p2)
    ref = oracle.boxfgt(t, t.fvals, delta, eps)
    r = ref.reshape(t.nboxes, -1)[lv]
    err = rel_l2(p.reshape(t.nboxes, -1)[lv], r)
    assert err < min(1e-6, 10 * eps), err
    # the split result is not the FP64 one (the selector took effect)
    hb.set_default_precision(hb.BFGT_PREC_FP64)
    q, _, _, _, _ = call(t, delta, eps)
    assert rel_l2(q.reshape(t.nboxes, -1)[lv], r) < 1e-11
    assert not np.array_equal(p, q)


def test_split_selected_falls_back_to_fp64_where_split_cannot_serve(trees):
    """eps = 1e-12 is below what split precision reaches: boxfgt_ runs it in FP64."""
    t = trees["ad_leg_per"]
    lv = t.leaves()
    hb.set_default_precision(hb.BFGT_PREC_SPLIT)
    p, _, _, _, _ = call(t, 1e-4, 1e-12)
    ref = oracle.boxfgt(t, t.fvals, 1e-4, 1e-12)
    assert rel_l2(p.reshape(t.nboxes, -1)[lv], ref.reshape(t.nboxes, -1)[lv]) < 1e-11


def test_zero_pot_is_cleared_on_the_device_not_uploaded(trees):
    """The reference's callers zero pot before each call (hpots2dadap.f:97-101,
    321-325).  A zero pot is then not uploaded: the call moves fvals up and pot
    down only, and gives the same bits as the upload path, which a single -0.0
    in pot forces (-0.0 is not skipped, so sums of signed zeros stay as the
    reference's)."""
    t = trees["ad16_leg_per"]
    lv = t.leaves()
    p0, _, _, _, _ = call(t, 1e-4, 1e-6)
    b0 = hb.last_call_bytes()
    leaf_bytes = 8 * t.npbox * len(lv)
    assert leaf_bytes <= b0["h2d"] < 2 * leaf_bytes  # fvals runs only
    assert b0["d2h"] >= leaf_bytes
    pot = np.zeros(t.npbox * t.nboxes)
    pot.reshape(t.nboxes, -1)[lv[0], 0] = -0.0
    ti = np.zeros(20)
    hb.boxfgt(1, 2, 1e-4, 1e-6, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree, t.itree.copy(),
              t.iptr, t.centers, t.boxsize, np.ascontiguousarray(t.fvals), 1, pot, None, None, 0, 0, None, 0, None,
              None, None, ti)
    b1 = hb.last_call_bytes()
    assert b1["h2d"] == b0["h2d"] + b0["d2h"]  # pot uploaded too
    np.testing.assert_array_equal(pot, p0)
    # a nonzero pot is accumulated into
    base = np.random.default_rng(5).standard_normal(t.npbox * t.nboxes)
    pot2 = base.copy()
    hb.boxfgt(1, 2, 1e-4, 1e-6, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree, t.itree.copy(),
              t.iptr, t.centers, t.boxsize, np.ascontiguousarray(t.fvals), 1, pot2, None, None, 0, 0, None, 0, None,
              None, None, ti)
    np.testing.assert_allclose(pot2.reshape(t.nboxes, -1)[lv], (base + p0).reshape(t.nboxes, -1)[lv], rtol=0,
                               atol=1e-14 * (np.abs(base).max() + np.abs(p0).max()))
    nonleaf = t.nchild() > 0
    np.testing.assert_array_equal(pot2.reshape(t.nboxes, -1)[nonleaf], base.reshape(t.nboxes, -1)[nonleaf])


def test_a_solver_step_cycle_stays_cached(trees):
    """One heat-solver step calls boxfgt once per delta (4 dt, and 4 (dt - t_q)
    for 4 Gauss nodes: hpots2dadap.f:79, 329-346); the next step repeats the
    cycle, which must then find all 5 plans."""
    t = trees["uni3_leg_per"]
    dt = 1e-3
    xq = (np.polynomial.legendre.leggauss(4)[0] + 1) / 2
    deltas = [4 * dt] + [4 * (1 - x) * dt for x in xq]
    first = [call(t, d, 1e-6)[0] for d in deltas]
    h0 = hb.plan_cache_info()["hits"]
    again = [call(t, d, 1e-6)[0] for d in deltas]
    info = hb.plan_cache_info()
    assert info["hits"] == h0 + len(deltas) and info["entries"] == len(deltas)
    for a, b in zip(first, again):
        np.testing.assert_array_equal(a, b)


def test_pageable_host_arrays_through_pinned_chunks():
    """Ordinary (pageable) host arrays, as a Fortran caller has them, are staged
    through the plan's pinned 8 MB chunks: on a tree whose leaf runs span
    several chunks (16,384 order-16 leaves, 33 MB per array) the result equals
    bit for bit the one from page-locked arrays, with a nonzero pot accumulated
    into as well."""
    import torch
    rng = np.random.default_rng(3)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (5, 2)), np.full(5, 0.05), rng.standard_normal(5))
    t = hb.build_uniform(7, g, norder=16, ipoly=0, iperiod=1)
    n = t.npbox * t.nboxes
    f_pg = np.ascontiguousarray(t.fvals).reshape(-1).copy()
    f_pin = torch.from_numpy(f_pg.copy()).pin_memory()
    base = np.random.default_rng(4).standard_normal(n)
    for start in (np.zeros(n), base):
        p_pg = start.copy()
        p_pin = torch.from_numpy(start.copy()).pin_memory()
        for fv, pv in ((f_pg, p_pg), (f_pin.numpy(), p_pin.numpy())):
            hb.boxfgt(1, 2, 1e-3, 1e-6, t.ipoly, t.iperiod, t.norder, t.npbox, t.nboxes, t.nlevels, t.ltree,
                      t.itree.copy(), t.iptr, t.centers, t.boxsize, fv, 1, pv, None, None, 0, 0, None, 0, None, None,
                      None, np.zeros(20))
        np.testing.assert_array_equal(p_pg, p_pin.numpy())
        assert not np.array_equal(p_pg, start)
