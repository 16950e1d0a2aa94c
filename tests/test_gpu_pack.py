"""Densities packed into the tensor-core MMA rows (split precision, nd > 1).

A chunk of ncol columns fills ncol*n rows per density, so a pass through its
steps carries min(nd, 128 / (ncol*n)) densities.  Each density of an
nd-density transform must equal the nd = 1 transform of that density alone:
the packed kernels do every density's arithmetic in the same order as the
unpacked ones, only in other MMA rows.  Checked for pot, grad and hess
(ifpgh = 3, whose eval stage packs 3 nd derivative densities).

The order-8 trees and deltas of the uneven-trees case give chunks of 1 to 16
columns (8 to 128 rows per density).  That makes the rarer cases occur:
8-row FP64 tiles of two densities in one warp; tiles whose densities fall in
different groups of shared-memory L slots; and passes of unequal size
(nd = 5).  Both nd variants are also checked against the oracle.
"""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle
from test_gpu_batch import leaf_values, rel_l2, uneven_trees

pytestmark = pytest.mark.gpu

# regime-B trees with chunks of 1..8 columns, and one periodic-Fourier tree
TREES = [0, 1, 2, 3, 7]


def run_pgh(plan, t, f, nd):
    import torch
    npb = t.npbox
    F = torch.from_numpy(np.ascontiguousarray(f).reshape(-1)).cuda()
    P = torch.zeros_like(F)
    G = torch.zeros(t.nboxes * npb * 2 * nd, dtype=torch.float64, device="cuda")
    H = torch.zeros(t.nboxes * npb * 3 * nd, dtype=torch.float64, device="cuda")
    plan.execute_pgh(3, F, P, G, H)
    plan.check()
    return (P.cpu().numpy().reshape(t.nboxes, npb, nd), G.cpu().numpy().reshape(t.nboxes, npb, 2, nd),
            H.cpu().numpy().reshape(t.nboxes, npb, 3, nd))


@pytest.mark.parametrize("nd", [5, 16])
def test_packed_densities_equal_single_density_transforms(nd):
    specs = uneven_trees(8, 6)
    for i in TREES:
        t, delta, eps, _, prec = specs[i]
        f = leaf_values(t, nd, 500 + i)
        packed = hb.Plan(t, delta, eps, nd=nd, precision=prec)
        single = hb.Plan(t, delta, eps, nd=1, precision=prec)
        p, g, h = run_pgh(packed, t, f, nd)
        lv = t.leaves()
        for k in range(nd):
            p1, g1, h1 = run_pgh(single, t, f[:, :, k:k + 1], 1)
            for got, ref, nm in ((p[..., k], p1[..., 0], "pot"), (g[..., k], g1[..., 0], "grad"),
                                 (h[..., k], h1[..., 0], "hess")):
                err = np.abs(got[lv] - ref[lv]).max() / max(np.abs(ref[lv]).max(), 1e-300)
                assert err <= 1e-13, (i, delta, nd, k, nm, err)
        # and the packed transform against the oracle
        ref = oracle.boxfgt(t, f, delta, eps, nd=nd).reshape(t.nboxes, -1)
        err = rel_l2(p.reshape(t.nboxes, -1)[lv], ref[lv])
        assert err <= 1e-6, (i, delta, nd, err)
        packed.close()
        single.close()
