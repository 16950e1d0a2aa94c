"""Quad trees in the reference's layout (common/tree_routs_nd.f:1626-1706) and
the caller-side generator of test and benchmark inputs (the vol_tree_build
criterion of common/tree_vol_coeffs_nd.f:440-780, built in libbfgt_b200.so).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class Tree:
    norder: int
    ipoly: int
    iperiod: int
    nboxes: int
    nlevels: int
    ltree: int
    itree: np.ndarray     # int32 (ltree,)
    iptr: np.ndarray      # int32 (8,)
    centers: np.ndarray   # float64 (nboxes, 2) == Fortran centers(2, nboxes)
    boxsize: np.ndarray   # float64 (nlevels+1,)
    fvals: np.ndarray = field(default=None)  # float64 (nboxes, npbox) == fvals(1, npbox, nboxes)

    # views of the itree arrays (1-based box ids, as in the reference)
    def laddr(self):
        return self.itree[: 2 * (self.nlevels + 1)].reshape(self.nlevels + 1, 2)

    def _seg(self, k, width=1):
        s = self.iptr[k] - 1
        return self.itree[s: s + width * self.nboxes]

    def ilevel(self):
        return self._seg(1)

    def iparent(self):
        return self._seg(2)

    def nchild(self):
        return self._seg(3)

    def ichild(self):
        return self._seg(4, 4).reshape(self.nboxes, 4)

    def ncoll(self):
        return self._seg(5)

    def coll(self):
        return self._seg(6, 9).reshape(self.nboxes, 9)

    def leaves(self):
        """0-based indices of the leaf boxes."""
        return np.nonzero(self.nchild() == 0)[0]

    @property
    def npbox(self):
        return self.norder * self.norder

    def copy(self):
        return Tree(self.norder, self.ipoly, self.iperiod, self.nboxes, self.nlevels, self.ltree, self.itree.copy(),
                    self.iptr.copy(), self.centers.copy(), self.boxsize.copy(),
                    None if self.fvals is None else self.fvals.copy())

    def grid_points(self, boxes=None):
        """Physical coordinates of the leaf grid points: (len(boxes), npbox, 2)."""
        from .nodes import leaf_nodes
        x, _, _, _ = leaf_nodes(self.ipoly, self.norder)
        n = self.norder
        if boxes is None:
            boxes = np.arange(self.nboxes)
        lev = self.ilevel()[boxes]
        h = self.boxsize[lev] / 2
        gx = np.tile(x, n)            # x index fastest
        gy = np.repeat(x, n)
        c = self.centers[boxes]
        return np.stack([c[:, 0:1] + gx[None, :] * h[:, None], c[:, 1:2] + gy[None, :] * h[:, None]], axis=-1)


def _export(h, norder, ipoly, iperiod) -> Tree:
    L = _lib.lib()
    nb, nl, lt = C.c_int(), C.c_int(), C.c_int()
    _lib.check(L.bfgt_tree_sizes(h, C.byref(nb), C.byref(nl), C.byref(lt)))
    nb, nl, lt = nb.value, nl.value, lt.value
    itree = np.zeros(lt, np.int32)
    iptr = np.zeros(8, np.int32)
    centers = np.zeros(2 * nb)
    boxsize = np.zeros(nl + 1)
    fvals = np.zeros(nb * norder * norder)
    _lib.check(L.bfgt_tree_export(h, itree, iptr, centers, boxsize, fvals))
    L.bfgt_tree_free(h)
    return Tree(norder, ipoly, iperiod, nb, nl, lt, itree, iptr, centers.reshape(nb, 2), boxsize,
                fvals.reshape(nb, norder * norder))


def gauss_params(centers, widths, amps) -> np.ndarray:
    g = np.stack([np.asarray(centers)[:, 0], np.asarray(centers)[:, 1], np.asarray(widths), np.asarray(amps)], 1)
    return np.ascontiguousarray(g, dtype=np.float64)


def build_adaptive(gauss, norder=16, ipoly=0, iperiod=1, eps=1e-10, boxlen=1.0, eta=1.0, minlev=0,
                   maxlev=0) -> Tree:
    """Adaptive 2:1-balanced tree resolving f = sum a exp(-|x-c|^2/w^2) (rows of gauss: cx, cy, w, a)."""
    L = _lib.lib()
    h = C.c_void_p()
    g = np.ascontiguousarray(gauss, dtype=np.float64).reshape(-1, 4)
    _lib.check(L.bfgt_tree_build_gauss(C.byref(h), int(ipoly), int(iperiod), float(eps), float(boxlen), int(norder),
                                       float(eta), int(g.shape[0]), g.reshape(-1), int(minlev), int(maxlev)))
    return _export(h, norder, ipoly, iperiod)


def build_uniform(nlev, gauss, norder=8, ipoly=0, iperiod=1, boxlen=1.0) -> Tree:
    """Uniform tree of depth nlev (4**nlev leaves) with f sampled on every box."""
    L = _lib.lib()
    h = C.c_void_p()
    g = np.ascontiguousarray(gauss, dtype=np.float64).reshape(-1, 4)
    _lib.check(L.bfgt_tree_build_uniform(C.byref(h), int(ipoly), int(iperiod), float(boxlen), int(norder),
                                         int(nlev), int(g.shape[0]), g.reshape(-1)))
    return _export(h, norder, ipoly, iperiod)
