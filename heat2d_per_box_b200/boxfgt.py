"""Python mirror of the reference's boxfgt interface (bfgt/boxfgt.f:5-8) over
the C ABI of libbfgt_b200.so, plus the device-resident plan.

`boxfgt(...)` takes the reference's argument list in order, with numpy arrays
in the reference layout, and calls the gfortran-ABI symbol boxfgt_ exactly as
compiled Fortran would (every argument by reference).  Like the reference it
accumulates into pot on leaf boxes and rewrites the colleague arrays of itree.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import BFGT_PREC_FP64, BFGT_PREC_SPLIT, BfgtError


def _iref(v):
    return C.byref(C.c_int(int(v)))


def _arr(a):
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
        raise TypeError("grad/hess/targs/pote/grade/hesse must be C-contiguous float64 numpy arrays")
    return a.ctypes.data


def boxfgt(nd, ndim, delta, eps, ipoly, iperiod, norder, npbox, nboxes, nlevels, ltree, itree, iptr, centers, boxsize,
           fvals, ifpgh, pot, grad, hess, ifnewtree, ntarg, targs, ifpghtarg, pote, grade, hesse, timeinfo):
    """Drop-in for `call boxfgt(...)`: pot(nd,npbox,nboxes) += G_delta * fvals on leaves
    (and grad(nd,2,npbox,nboxes), hess(nd,3,npbox,nboxes) for ifpgh = 2, 3).

    Raises BfgtError when the library records an error (the Fortran routine
    itself has no error argument; the C ABI keeps its message in
    bfgt_last_error()).
    """
    L = _lib.lib()
    for name, a, dt in (("itree", itree, np.int32), ("iptr", iptr, np.int32), ("centers", centers, np.float64),
                        ("boxsize", boxsize, np.float64), ("fvals", fvals, np.float64), ("pot", pot, np.float64),
                        ("timeinfo", timeinfo, np.float64)):
        if not (isinstance(a, np.ndarray) and a.dtype == dt and a.flags.c_contiguous):
            raise TypeError(f"{name} must be a C-contiguous {np.dtype(dt).name} numpy array")
    ip = C.c_int(int(iperiod))
    nb, nl, lt = C.c_int(int(nboxes)), C.c_int(int(nlevels)), C.c_int(int(ltree))
    dl, ep = C.c_double(float(delta)), C.c_double(float(eps))
    L.boxfgt_(_iref(nd), _iref(ndim), C.byref(dl), C.byref(ep), _iref(ipoly), C.byref(ip), _iref(norder), _iref(npbox),
              C.byref(nb), C.byref(nl), C.byref(lt), itree.reshape(-1), iptr, centers.reshape(-1), boxsize,
              fvals.reshape(-1), _iref(ifpgh), pot.reshape(-1), _arr(grad), _arr(hess), _iref(ifnewtree), _iref(ntarg),
              _arr(targs), _iref(ifpghtarg), _arr(pote), _arr(grade), _arr(hesse), timeinfo)
    err = _lib.last_error()
    if err:
        raise BfgtError(1, err)
    return pot


def set_default_precision(precision):
    """Precision mode of the drop-in boxfgt (BFGT_PREC_FP64 or BFGT_PREC_SPLIT)."""
    _lib.check(_lib.lib().bfgt_set_default_precision(int(precision)))


def plan_cache_info():
    """The drop-in entry points' plan cache: entries, capacity, hits, misses."""
    out = np.zeros(4, np.int64)
    _lib.check(_lib.lib().bfgt_plan_cache_info(out.ctypes.data))
    return {"entries": int(out[0]), "capacity": int(out[1]), "hits": int(out[2]), "misses": int(out[3])}


def last_call_bytes():
    """Host-to-device and device-to-host bytes of the last boxfgt_ call (pot
    runs that were all zero on the host are cleared on the device, not
    uploaded)."""
    out = np.zeros(2, np.float64)
    _lib.check(_lib.lib().bfgt_boxfgt_last_bytes(out.ctypes.data))
    return {"h2d": int(out[0]), "d2h": int(out[1])}


def plan_cache_clear():
    """Frees the plans the drop-in entry points keep."""
    _lib.check(_lib.lib().bfgt_plan_cache_clear())


class Plan:
    """Device-resident boxfgt for one tree / delta / eps / norder / nd.

    execute(d_fvals, d_pot, stream) takes raw device pointers (ints) or torch
    CUDA tensors; execute_host(fvals, pot) takes host numpy arrays.
    """

    def __init__(self, tree, delta, eps, nd=1, precision=BFGT_PREC_FP64):
        self._L = _lib.lib()
        self.tree = tree
        self.nd = nd
        self.itree = tree.itree.copy()
        h = C.c_void_p()
        _lib.check(self._L.bfgt_plan_create(C.byref(h), int(nd), float(delta), float(eps), int(tree.ipoly),
                                            int(tree.iperiod), int(tree.norder), int(tree.nboxes), int(tree.nlevels),
                                            int(tree.ltree), self.itree, np.ascontiguousarray(tree.iptr, np.int32),
                                            np.ascontiguousarray(tree.centers, np.float64).reshape(-1),
                                            np.ascontiguousarray(tree.boxsize, np.float64), int(precision)))
        self._h = h

    @staticmethod
    def _ptr(x):
        if x is None:
            return None
        if isinstance(x, int):
            return x
        if hasattr(x, "data_ptr"):
            return x.data_ptr()
        raise TypeError("expected a device pointer or a torch CUDA tensor")

    def execute(self, d_fvals, d_pot, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute(self._h, self._ptr(d_fvals), self._ptr(d_pot), s))

    def execute_noalloc(self, d_fvals, d_pot, stream=None):
        """Same transform as execute(), with no device allocation: the plane-wave
        scratch comes from the library's static per-GPU array (see bfgt.h)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_noalloc(self._h, self._ptr(d_fvals), self._ptr(d_pot), s))

    def noalloc_need(self):
        v = C.c_size_t()
        _lib.check(self._L.bfgt_plan_noalloc_need(self._h, C.byref(v)))
        return int(v.value)

    def execute_host(self, fvals, pot, stream=None):
        fv = np.ascontiguousarray(fvals, np.float64)
        if not (isinstance(pot, np.ndarray) and pot.dtype == np.float64 and pot.flags.c_contiguous):
            raise TypeError("pot must be a C-contiguous float64 array")
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_host(self._h, fv.ctypes.data, pot.ctypes.data, s))
        return pot

    def execute_pgh(self, ifpgh, d_fvals, d_pot, d_grad=None, d_hess=None, stream=None):
        """pot += K f; grad(nd,2,npbox,nboxes) and hess(nd,3,npbox,nboxes) (xx, xy, yy)
        += its derivatives for ifpgh = 2, 3 (device arrays)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_pgh(self._h, int(ifpgh), self._ptr(d_fvals), self._ptr(d_pot),
                                                 self._ptr(d_grad), self._ptr(d_hess), s))

    def execute_pgh_host(self, ifpgh, fvals, pot, grad=None, hess=None, stream=None):
        fv = np.ascontiguousarray(fvals, np.float64)
        for nm, a in (("pot", pot), ("grad", grad), ("hess", hess)):
            if a is not None and not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError(f"{nm} must be a C-contiguous float64 array")
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_pgh_host(self._h, int(ifpgh), fv.ctypes.data, pot.ctypes.data,
                                                      None if grad is None else grad.ctypes.data,
                                                      None if hess is None else hess.ctypes.data, s))
        return pot, grad, hess

    def eval_targets(self, ncomp, d_vals, ntarg, d_targs, d_out, stream=None):
        """out(nd*ncomp, ntarg) = leaf interpolants of vals(nd*ncomp, npbox, nboxes) at targs(2, ntarg)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_eval_targets(self._h, int(ncomp), self._ptr(d_vals), int(ntarg),
                                                  self._ptr(d_targs), self._ptr(d_out), s))

    def execute_adjoint(self, d_potbar, d_fbar, stream=None):
        """fbar += K^T potbar on leaf boxes (the transpose of execute: pot += K fvals)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_adjoint(self._h, self._ptr(d_potbar), self._ptr(d_fbar), s))

    def execute_adjoint_host(self, potbar, fbar, stream=None):
        pb = np.ascontiguousarray(potbar, np.float64)
        if not (isinstance(fbar, np.ndarray) and fbar.dtype == np.float64 and fbar.flags.c_contiguous):
            raise TypeError("fbar must be a C-contiguous float64 array")
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_execute_adjoint_host(self._h, pb.ctypes.data, fbar.ctypes.data, s))
        return fbar

    def graph_capture(self, d_fvals, d_pot, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_graph_capture(self._h, self._ptr(d_fvals), self._ptr(d_pot), s))

    def graph_launch(self, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_plan_graph_launch(self._h, s))

    def set_wait_limit(self, polls=None):
        """Poll limit of the bounded device waits (None restores the default)."""
        _lib.check(self._L.bfgt_plan_set_wait_limit(self._h, 0xFFFFFFFF if polls is None else int(polls)))

    def autotune(self, stream=None):
        """Times the plan's compiled kernel shapes on its own work and keeps the
        fastest (see bfgt_plan_autotune): FP64 tile shapes, or the split
        kernels' Y staging, x tiles and eval step groups.  Tune a plan before
        putting it in a Batch (a batch keeps the shapes its plans had when it
        was created).  Returns (form ms, eval ms, shapes timed)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        rep = np.zeros(4)
        _lib.check(self._L.bfgt_plan_autotune(self._h, s, rep))
        return float(rep[0]), float(rep[1]), int(rep[2] + rep[3])

    def check(self):
        """Waits for the device; raises BfgtError if a bounded device wait timed out."""
        _lib.check(self._L.bfgt_plan_check(self._h))

    def stage_ms(self):
        """Per-stage device ms summed over the executes since the last call (see bfgt_plan_stage_ms)."""
        out = np.zeros(8)
        _lib.check(self._L.bfgt_plan_stage_ms(self._h, out))
        return out

    def reserve_events(self, n):
        _lib.check(self._L.bfgt_plan_reserve_events(self._h, int(n)))

    def info(self):
        out = np.zeros(16, np.int32)
        _lib.check(self._L.bfgt_plan_info(self._h, out))
        keys = ["npwlevel", "npw", "nlevstart", "nlevend", "regime", "nleafbox", "npwleaves", "nnear_targets",
                "nnear_pairs", "mnlist1", "iperiod_int", "nchunks", "launches", "form_tile", "eval_tile",
                "split_shape"]
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def work(self):
        out = np.zeros(16)
        _lib.check(self._L.bfgt_plan_work(self._h, out))
        keys = ["flops", "bytes", "tc_flops", "points", "flops_form", "flops_eval", "flops_near", "flops_translate",
                "bytes_form", "bytes_eval", "bytes_near", "tc_flops_form", "tc_flops_eval", "host_h2d_bytes",
                "host_d2h_bytes"]
        return {k: float(out[i]) for i, k in enumerate(keys)}

    def close(self):
        if getattr(self, "_h", None):
            self._L.bfgt_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Transforms of several plans run together (bfgt_batch_* in bfgt.h).

    The leaf arrays of the plans are packed one after another: plan i's
    fvals/pot occupy elements offsets[i]:offsets[i+1] of the batch arrays.
    The plans must stay open while the batch exists.
    """

    def __init__(self, plans):
        self._L = _lib.lib()
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = C.c_void_p()
        _lib.check(self._L.bfgt_batch_create(C.byref(h), len(self.plans), C.cast(arr, C.c_void_p)))
        self._h = h
        off = np.zeros(len(self.plans) + 1, np.int64)
        _lib.check(self._L.bfgt_batch_layout(self._h, off.ctypes.data))
        self.offsets = off

    def execute(self, d_fvals, d_pot, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_batch_execute(self._h, Plan._ptr(d_fvals), Plan._ptr(d_pot), s))

    def execute_adjoint(self, d_potbar, d_fbar, stream=None):
        """fbar += K_i^T potbar for every plan i (packed arrays, same layout)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_batch_execute_adjoint(self._h, Plan._ptr(d_potbar), Plan._ptr(d_fbar), s))

    def graph_capture(self, d_fvals, d_pot, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_batch_graph_capture(self._h, Plan._ptr(d_fvals), Plan._ptr(d_pot), s))

    def graph_launch(self, stream=None):
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        _lib.check(self._L.bfgt_batch_graph_launch(self._h, s))

    def stage_ms(self):
        out = np.zeros(8)
        _lib.check(self._L.bfgt_batch_stage_ms(self._h, out))
        return out

    def info(self):
        out = np.zeros(8, np.int32)
        _lib.check(self._L.bfgt_batch_info(self._h, out))
        keys = ["plans", "launches", "form_items", "eval_items", "translate_blocks", "near_blocks"]
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def check(self):
        _lib.check(self._L.bfgt_batch_check(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.bfgt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_plan_dump(tree, delta, eps, nd=1, mnlist1_cap=64):
    """Host half of a plan (no device needed): lists, band patterns, near-field tables, PW nodes."""
    L = _lib.lib()
    n, nb, nl = tree.norder, tree.nboxes, tree.nlevels
    it = tree.itree.copy()
    info = np.zeros(16, np.int32)
    out = dict(ifpwexp=np.zeros(nb, np.int32), nlist1=np.zeros(nb, np.int32),
               list1=np.zeros(mnlist1_cap * nb, np.int32), nlistpw=np.zeros(nb, np.int32),
               listpw=np.zeros(8 * nb, np.int32), ind_loc=np.zeros(2 * (n + 1) * 13 * (nl + 1), np.int32),
               tab_loc=np.zeros(n * n * 13 * (nl + 1)), ts=np.zeros(256), ws=np.zeros(256))
    _lib.check(L.bfgt_host_plan_dump(int(nd), float(delta), float(eps), int(tree.ipoly), int(tree.iperiod), int(n),
                                     int(nb), int(nl), int(tree.ltree), it, np.ascontiguousarray(tree.iptr, np.int32),
                                     np.ascontiguousarray(tree.centers, np.float64).reshape(-1),
                                     np.ascontiguousarray(tree.boxsize, np.float64), info.ctypes.data,
                                     out["ifpwexp"].ctypes.data, out["nlist1"].ctypes.data, out["list1"].ctypes.data,
                                     int(mnlist1_cap), out["nlistpw"].ctypes.data, out["listpw"].ctypes.data,
                                     out["ind_loc"].ctypes.data, out["tab_loc"].ctypes.data, out["ts"].ctypes.data,
                                     out["ws"].ctypes.data))
    keys = ["npwlevel", "npw", "nlevstart", "nlevend", "regime", "nleafbox", "npwleaves", "nnear_targets",
            "nnear_pairs", "mnlist1", "iperiod_int", "nchunks"]
    d = {k: int(info[i]) for i, k in enumerate(keys)}
    out["list1"] = out["list1"].reshape(nb, mnlist1_cap)
    out["listpw"] = out["listpw"].reshape(nb, 8)
    out["ts"] = out["ts"][: d["npw"]].copy()
    out["ws"] = out["ws"][: d["npw"]].copy()
    out["itree"] = it
    return d, out
