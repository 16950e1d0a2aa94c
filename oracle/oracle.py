"""ctypes binding of the CPU oracle (oracle/bfgt_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's CPU-baseline leg.  It restates the reference's
boxfgt (bfgt/boxfgt.f:5-1591, ndim=2, ifpgh=1, 2, 3) in C.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import build as _build

_lib = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class _Info(C.Structure):
    _fields_ = [
        ("npwlevel", C.c_int), ("npwlevel_int", C.c_int), ("npw", C.c_int), ("nlevstart", C.c_int),
        ("nlevend", C.c_int), ("iperiod_int", C.c_int), ("regime", C.c_int), ("mnlist1", C.c_int),
        ("nleafbox", C.c_int),
        ("ifpwexp", C.POINTER(C.c_int)), ("nlist1", C.POINTER(C.c_int)), ("list1", C.POINTER(C.c_int)),
        ("mnlist1_cap", C.c_int), ("nlistpw", C.POINTER(C.c_int)), ("listpw", C.POINTER(C.c_int)),
        ("ind_loc", C.POINTER(C.c_int)), ("tab_loc", C.POINTER(C.c_double)), ("ts", C.POINTER(C.c_double)),
        ("ws", C.POINTER(C.c_double)),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(str(path))
        L.oracle_boxfgt.restype = None
        L.oracle_boxfgt.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, C.c_void_p, C.c_void_p]
        L.oracle_boxfgt_pgh.restype = None
        L.oracle_boxfgt_pgh.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, _f64p, C.c_void_p,
                                        C.c_void_p]
        L.oracle_eval_targets.restype = None
        L.oracle_eval_targets.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                          _f64p, C.c_int, _f64p, _f64p, C.c_void_p]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_nodes.argtypes = [C.c_int, C.c_int, _f64p, _f64p, _f64p, _f64p]
        L.oracle_gauss_legendre.argtypes = [C.c_int, _f64p, _f64p]
        L.oracle_pw_tables.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_double, C.c_double, _f64p, _f64p]
        L.oracle_besseljs.argtypes = [C.c_int, C.c_double, _f64p]
        _lib = L
    return _lib


@dataclass
class OracleInfo:
    npwlevel: int
    npwlevel_int: int
    npw: int
    nlevstart: int
    nlevend: int
    iperiod_int: int
    regime: int
    mnlist1: int
    nleafbox: int
    ifpwexp: np.ndarray
    nlist1: np.ndarray
    list1: np.ndarray
    nlistpw: np.ndarray
    listpw: np.ndarray
    ind_loc: np.ndarray
    tab_loc: np.ndarray
    ts: np.ndarray
    ws: np.ndarray


def boxfgt(tree, fvals, delta, eps, nd=1, pot=None, itree=None, timeinfo=None, with_info=False, threads=0):
    """Runs the oracle; returns pot (accumulated into a copy of `pot` or zeros).

    tree: a heat2d_per_box_b200.tree.Tree (or any object with the same fields).
    fvals: (nboxes, npbox, nd)-shaped or flat array in the reference layout
    fvals(nd, npbox, nboxes).  itree is rewritten (colleagues) as the
    reference does; a copy of tree.itree is used unless itree is given.
    """
    L = lib()
    if threads:
        L.oracle_set_threads(int(threads))
    n = tree.norder
    fv = np.ascontiguousarray(fvals, dtype=np.float64).reshape(-1)
    out = np.zeros(nd * n * n * tree.nboxes) if pot is None else np.array(pot, dtype=np.float64).reshape(-1).copy()
    it = np.array(tree.itree if itree is None else itree, dtype=np.int32).copy()
    ti = np.zeros(20) if timeinfo is None else timeinfo
    info = None
    keep = []
    if with_info:
        nb, nl = tree.nboxes, tree.nlevels
        cap = 64
        arrs = dict(
            ifpwexp=np.zeros(nb, np.int32), nlist1=np.zeros(nb, np.int32), list1=np.zeros(cap * nb, np.int32),
            nlistpw=np.zeros(nb, np.int32), listpw=np.zeros(8 * nb, np.int32),
            ind_loc=np.zeros(2 * (n + 1) * 13 * (nl + 1), np.int32), tab_loc=np.zeros(n * n * 13 * (nl + 1)),
            ts=np.zeros(256), ws=np.zeros(256))
        keep.append(arrs)
        info = _Info()
        for k in ("ifpwexp", "nlist1", "list1", "nlistpw", "listpw", "ind_loc"):
            setattr(info, k, arrs[k].ctypes.data_as(C.POINTER(C.c_int)))
        for k in ("tab_loc", "ts", "ws"):
            setattr(info, k, arrs[k].ctypes.data_as(C.POINTER(C.c_double)))
        info.mnlist1_cap = cap
    L.oracle_boxfgt(int(nd), float(delta), float(eps), int(tree.ipoly), int(tree.iperiod), int(n), int(tree.nboxes),
                    int(tree.nlevels), it, np.ascontiguousarray(tree.iptr, dtype=np.int32),
                    np.ascontiguousarray(tree.centers, dtype=np.float64).reshape(-1),
                    np.ascontiguousarray(tree.boxsize, dtype=np.float64), fv, out,
                    ti.ctypes.data, C.addressof(info) if info is not None else None)
    if not with_info:
        return out
    a = keep[0]
    oi = OracleInfo(info.npwlevel, info.npwlevel_int, info.npw, info.nlevstart, info.nlevend, info.iperiod_int,
                    info.regime, info.mnlist1, info.nleafbox, a["ifpwexp"], a["nlist1"],
                    a["list1"].reshape(tree.nboxes, 64), a["nlistpw"], a["listpw"].reshape(tree.nboxes, 8),
                    a["ind_loc"], a["tab_loc"], a["ts"][: info.npw].copy(), a["ws"][: info.npw].copy())
    return out, oi, it


def boxfgt_pgh(tree, fvals, delta, eps, ifpgh, nd=1, threads=0):
    """Runs the oracle with ifpgh = 1, 2 or 3; returns (pot, grad, hess) in the
    reference layouts pot(nd,npbox,nboxes), grad(nd,2,npbox,nboxes),
    hess(nd,3,npbox,nboxes) (xx, xy, yy), flattened; grad/hess are None below
    ifpgh 2/3."""
    L = lib()
    if threads:
        L.oracle_set_threads(int(threads))
    n = tree.norder
    m = nd * n * n * tree.nboxes
    fv = np.ascontiguousarray(fvals, dtype=np.float64).reshape(-1)
    pot = np.zeros(m)
    grad = np.zeros(2 * m) if ifpgh >= 2 else None
    hess = np.zeros(3 * m) if ifpgh == 3 else None
    it = np.array(tree.itree, dtype=np.int32).copy()
    L.oracle_boxfgt_pgh(int(nd), float(delta), float(eps), int(tree.ipoly), int(tree.iperiod), int(n),
                        int(tree.nboxes), int(tree.nlevels), it, np.ascontiguousarray(tree.iptr, dtype=np.int32),
                        np.ascontiguousarray(tree.centers, dtype=np.float64).reshape(-1),
                        np.ascontiguousarray(tree.boxsize, dtype=np.float64), fv, int(ifpgh), pot,
                        None if grad is None else grad.ctypes.data, None if hess is None else hess.ctypes.data)
    return pot, grad, hess


def eval_targets(tree, vals, targs, nd=1, itree=None):
    """Leaf interpolant of vals(nd, npbox, nboxes) at targets (ntarg, 2), as the
    reference's step 11 does (treedata_trans_nd + treedata_evalt_nd with
    pts_tree_sort).  Returns (out (ntarg, nd), 1-based leaf box per target).
    itree: the tree array after boxfgt rewrote its colleagues (the sort only
    reads levels, children and centers, so tree.itree works as well)."""
    L = lib()
    t = np.ascontiguousarray(targs, dtype=np.float64).reshape(-1, 2)
    nt = t.shape[0]
    out = np.zeros(nd * max(nt, 1))
    leaf = np.zeros(max(nt, 1), np.int32)
    it = np.ascontiguousarray(tree.itree if itree is None else itree, dtype=np.int32)
    L.oracle_eval_targets(int(nd), int(tree.ipoly), int(tree.norder), int(tree.nboxes), int(tree.nlevels), it,
                          np.ascontiguousarray(tree.iptr, dtype=np.int32),
                          np.ascontiguousarray(tree.centers, dtype=np.float64).reshape(-1),
                          np.ascontiguousarray(tree.boxsize, dtype=np.float64),
                          np.ascontiguousarray(vals, dtype=np.float64).reshape(-1), int(nt), t.reshape(-1), out,
                          leaf.ctypes.data)
    return out[: nd * nt].reshape(nt, nd), leaf[:nt]


def nodes(ipoly, n):
    """Leaf nodes, values->coefficients matrix u, coefficients->values v, weights (Fortran order)."""
    x, u, v, w = np.zeros(n), np.zeros(n * n), np.zeros(n * n), np.zeros(n)
    lib().oracle_nodes(int(ipoly), int(n), x, u, v, w)
    return x, u.reshape(n, n, order="F"), v.reshape(n, n, order="F"), w


def gauss_legendre(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().oracle_gauss_legendre(int(n), x, w)
    return x, w


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return int(lib().oracle_max_threads())
