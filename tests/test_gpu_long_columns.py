"""Coarse cutoff levels.  In the periodic-Fourier regime (delta = 1e-2) the
whole box is one cutoff box, so a uniform level-7 order-8 tree has 128 columns
of 128 leaves.  To keep the GPU busy, two things happen at plan creation:
- the split plan cuts its 8 chunks of 128 steps into step ranges;
- the FP64 plan cuts its 128-leaf columns into 16-leaf sub-columns, 4 to a
  chunk.
Each piece is summed like a separate chunk, so both plans must still match the
oracle (FP64 to 1e-11, split to 1e-6), for one and for two densities (packed
passes over pieces).  The chunk counts show that the cuts happened.
"""
import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from oracle import oracle
from test_gpu_batch import leaf_values, rel_l2

from conftest import gauss_sum

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nd", [1, 2])
@pytest.mark.parametrize("precision,bar", [(hb.BFGT_PREC_SPLIT, 1e-6), (hb.BFGT_PREC_FP64, 1e-11)])
def test_long_columns_cut_match_oracle(nd, precision, bar):
    import torch
    t = hb.build_uniform(7, gauss_sum(1, 3, 0.05, 0.1), norder=8, ipoly=0, iperiod=1)
    delta, eps = 1e-2, 1e-6 if precision == hb.BFGT_PREC_SPLIT else 1e-9
    f = leaf_values(t, nd, 700 + nd)
    plan = hb.Plan(t, delta, eps, nd=nd, precision=precision)
    info = plan.info()
    assert info["regime"] == 0 and info["nlevstart"] == 0
    if precision == hb.BFGT_PREC_SPLIT:
        assert info["nchunks"] > 8          # 8 chunks of 16 columns, cut into step ranges
    else:
        assert info["nchunks"] == 2 * 128   # 128-leaf columns: two chunks of 4 sub-columns each
    F = torch.from_numpy(f.reshape(-1)).cuda()
    P = torch.zeros_like(F)
    plan.execute(F, P)
    plan.check()
    got = P.cpu().numpy().reshape(t.nboxes, -1)
    ref = oracle.boxfgt(t, f, delta, eps, nd=nd).reshape(t.nboxes, -1)
    lv = t.leaves()
    err = rel_l2(got[lv], ref[lv])
    plan.close()
    assert err <= bar, (nd, precision, err)
