import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def gauss_sum(seed, ng, wlo, whi, amp="uniform", log_width=False):
    import heat2d_per_box_b200 as hb
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.5, 0.5, (ng, 2))
    w = np.exp(rng.uniform(np.log(wlo), np.log(whi), ng)) if log_width else rng.uniform(wlo, whi, ng)
    a = rng.uniform(-1, 1, ng) if amp == "uniform" else rng.standard_normal(ng)
    return hb.gauss_params(c, w, a)


@pytest.fixture(scope="session")
def trees():
    """Small trees covering uniform/adaptive, Legendre/Chebyshev, periodic/free."""
    import heat2d_per_box_b200 as hb
    out = {}
    g3 = gauss_sum(1, 3, 0.05, 0.1)
    out["uni3_leg_per"] = hb.build_uniform(3, g3, norder=8, ipoly=0, iperiod=1)
    out["uni3_cheb_per"] = hb.build_uniform(3, g3, norder=8, ipoly=1, iperiod=1)
    out["uni3_leg_free"] = hb.build_uniform(3, g3, norder=8, ipoly=0, iperiod=0)
    g6 = gauss_sum(2, 6, 0.01, 0.05, amp="normal", log_width=True)
    out["ad_leg_per"] = hb.build_adaptive(g6, norder=8, ipoly=0, iperiod=1, eps=1e-6, maxlev=6)
    out["ad_cheb_free"] = hb.build_adaptive(g6, norder=8, ipoly=1, iperiod=0, eps=1e-6, maxlev=6)
    out["ad16_leg_per"] = hb.build_adaptive(g6, norder=16, ipoly=0, iperiod=1, eps=1e-8, maxlev=5)
    # a tree with a leaf at level 1 and deep refinement elsewhere: reaches the
    # periodic level-1 image path of the near field
    # (with periodic wrap any depth-3 refinement splits every level-1 box, so
    # the path needs a depth-2 tree whose cutoff is level 2)
    g1 = hb.gauss_params(np.array([[0.25, 0.25]]), np.array([0.05]), np.array([1.0]))
    out["lev1_leaf_per"] = hb.build_adaptive(g1, norder=8, ipoly=0, iperiod=1, eps=1e-6, minlev=1, maxlev=2)
    return out
