"""Independent FP64 oracle: direct quadrature of the (periodic) Gaussian
convolution of the per-leaf polynomial interpolant.

TEST INFRASTRUCTURE ONLY.  It does not follow the reference's algorithm; it
evaluates, for every leaf grid point x,
    pot(x) = sum_{leaves B} sum_{images m} int_B exp(-|x - y - m L|^2/delta) p_B(y) dy
with p_B the tensor interpolant of the leaf values on B, by composite
Gauss-Legendre quadrature fine enough to resolve the Gaussian.  The transform
the reference computes (bfgt/boxfgt.f) approximates exactly this sum to a
relative error eps, so it checks the oracle's restatement end to end.
Use on small trees only.
"""
from __future__ import annotations

import numpy as np


def _nodes(ipoly, n):
    if ipoly == 0:
        x, _ = np.polynomial.legendre.leggauss(n)
        V = np.polynomial.legendre.legvander(x, n - 1)
        vand = lambda t: np.polynomial.legendre.legvander(t, n - 1)  # noqa: E731
    else:
        i = np.arange(1, n + 1)
        x = np.cos((2 * i - 1) * np.pi / (2 * n))[::-1].copy()
        V = np.polynomial.chebyshev.chebvander(x, n - 1)
        vand = lambda t: np.polynomial.chebyshev.chebvander(t, n - 1)  # noqa: E731
    return x, np.linalg.inv(V), vand


def direct_pot(tree, fvals, delta, nd=1, nq=16):
    """pot(nd, npbox, nboxes) on leaf boxes (zeros elsewhere), layout of the reference."""
    return direct_pgh(tree, fvals, delta, nd=nd, nq=nq, ifpgh=1)[0]


def direct_pgh(tree, fvals, delta, nd=1, nq=16, ifpgh=1):
    """(pot, grad, hess) on leaf boxes in the reference layouts pot(nd,npbox,nboxes),
    grad(nd,2,npbox,nboxes), hess(nd,3,npbox,nboxes) (xx, xy, yy), flattened;
    grad/hess are None below ifpgh 2/3.  Derivatives act on the target point:
    d/dx exp(-d^2/delta) = -2 d/delta exp(-d^2/delta), d^2/dx^2 adds
    (4 d^2/delta^2 - 2/delta)."""
    n = tree.norder
    npb = n * n
    x, U, vand = _nodes(tree.ipoly, n)
    gq, wq = np.polynomial.legendre.leggauss(nq)
    nch = np.asarray(tree.nchild())
    lev = np.asarray(tree.ilevel())
    leaves = np.nonzero(nch == 0)[0]
    L = float(tree.boxsize[0])
    fv = np.asarray(fvals, dtype=np.float64).reshape(tree.nboxes, npb, nd)
    # target coordinates
    h = tree.boxsize[lev[leaves]] / 2
    cx = tree.centers[leaves, 0][:, None] + x[None, :] * h[:, None]
    cy = tree.centers[leaves, 1][:, None] + x[None, :] * h[:, None]
    ux, ixinv = np.unique(cx.reshape(-1), return_inverse=True)
    uy, iyinv = np.unique(cy.reshape(-1), return_inverse=True)
    ixinv = ixinv.reshape(len(leaves), n)
    iyinv = iyinv.reshape(len(leaves), n)
    # target index arrays over (leaf, k1, k2), k1 fastest
    tix = np.repeat(ixinv[:, None, :], n, axis=1).reshape(len(leaves), npb)   # [leaf, k2*n+k1] -> x idx of k1
    tiy = np.repeat(iyinv[:, :, None], n, axis=2).reshape(len(leaves), npb)   # y idx of k2
    out = np.zeros((tree.nboxes, npb, nd))
    reach = np.sqrt(delta * 45.0)
    M = int(np.ceil((reach + L) / L)) if tree.iperiod == 1 else 0
    comps = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)][: {1: 1, 2: 3, 3: 6}[ifpgh]]
    orders = {1: 1, 2: 2, 3: 3}[ifpgh]
    acc = [np.zeros((len(leaves), npb, nd)) for _ in comps]
    for B in leaves:
        D = tree.boxsize[lev[B]]
        c = tree.centers[B]
        nsub = max(1, int(np.ceil(D / (0.25 * np.sqrt(delta)))))
        edges = np.linspace(-1, 1, nsub + 1)
        t = ((edges[:-1, None] + edges[1:, None]) / 2 + (edges[1:, None] - edges[:-1, None]) / 2 * gq[None, :]).reshape(-1)
        w = (np.repeat((edges[1:] - edges[:-1]) / 2, nq) * np.tile(wq, nsub)) * (D / 2)
        lag = vand(t) @ U            # (nquad, n): Lagrange basis at t
        lw = lag * w[:, None]

        def integ(u, cc, order):
            y = cc + t * D / 2
            tot = np.zeros((len(u), n))
            for m in range(-M, M + 1):
                d = u[:, None] - y[None, :] - m * L
                K = np.exp(-(d * d) / delta)
                if order == 1:
                    K = K * (-2 * d / delta)
                elif order == 2:
                    K = K * (4 * d * d / delta ** 2 - 2 / delta)
                tot += K @ lw
            return tot

        I = {(ax, o): integ(ux if ax == 0 else uy, c[ax], o) for ax in (0, 1) for o in range(orders)}
        F = fv[B].reshape(n, n, nd)   # [k2][k1][ind]
        for ind in range(nd):
            Fm = F[:, :, ind].T       # [i=x][j=y]
            for q, (ox, oy) in enumerate(comps):
                A = I[(0, ox)] @ Fm   # (X, n): sum_i Ix[x,i] F[i,j]
                acc[q][:, :, ind] += np.einsum("tpj,tpj->tp", A[tix], I[(1, oy)][tiy])
    res = []
    for q in range(len(comps)):
        o = np.zeros((tree.nboxes, npb, nd))
        o[leaves] = acc[q]
        res.append(o)
    # C order of the Fortran arrays: (nboxes, npbox, ncomp, nd)
    pot = res[0].reshape(-1)
    grad = np.stack([res[1], res[2]], axis=2).reshape(-1) if ifpgh >= 2 else None
    hess = np.stack([res[3], res[4], res[5]], axis=2).reshape(-1) if ifpgh == 3 else None
    return pot, grad, hess
