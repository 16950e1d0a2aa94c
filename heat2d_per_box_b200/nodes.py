"""Leaf node families (numpy): Gauss-Legendre (ipoly=0) and Chebyshev points of
the first kind (ipoly=1), ascending on [-1,1], as common/legeexps.f:141 and
common/chebexps.f:12 lay them out.  Used for grid coordinates in harnesses."""
from __future__ import annotations

import numpy as np


def leaf_nodes(ipoly: int, n: int):
    """Returns (x, u, v, w): nodes, values->coefficients, coefficients->values, weights."""
    if ipoly == 0:
        x, w = np.polynomial.legendre.leggauss(n)
        v = np.polynomial.legendre.legvander(x, n - 1)
    else:
        i = np.arange(1, n + 1)
        x = np.cos((2 * i - 1) * np.pi / (2 * n))[::-1].copy()
        v = np.polynomial.chebyshev.chebvander(x, n - 1)
        w = None
    u = np.linalg.inv(v)
    return x, u, v, w
