"""Generates tests/golden/golden.json: leaf-point values of the box FGT on small
trees, computed by the independent direct-quadrature oracle (oracle/quad.py),
which integrates the Gaussian against each leaf's interpolant without any of
the reference's approximations.  The analytic Fourier-mode case follows the
reference's known-answer test hpots/test_initpot.f:58-80,239-250 (periodic,
Chebyshev order 8, dt = 1e-5, delta = 4 dt, eps = 1e-9).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import heat2d_per_box_b200 as hb  # noqa: E402
from oracle import quad  # noqa: E402


def gauss(seed, ng, wlo, whi, normal=False, logw=False):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.5, 0.5, (ng, 2))
    w = np.exp(rng.uniform(np.log(wlo), np.log(whi), ng)) if logw else rng.uniform(wlo, whi, ng)
    a = rng.standard_normal(ng) if normal else rng.uniform(-1, 1, ng)
    return hb.gauss_params(c, w, a)


CASES = [
    dict(name="initpot_kat", kind="uniform", level=5, norder=8, ipoly=1, iperiod=1, delta=4e-5, eps=1e-9,
         density="fourier22", gauss=np.zeros((1, 4)).tolist()),
    dict(name="c1_stats_small", kind="uniform", level=3, norder=8, ipoly=0, iperiod=1, delta=1e-3, eps=1e-9,
         gauss=gauss(1, 3, 0.05, 0.1).tolist()),
    dict(name="periodic_fourier_regime", kind="uniform", level=3, norder=8, ipoly=1, iperiod=1, delta=1e-2,
         eps=1e-6, gauss=gauss(3, 4, 0.05, 0.1).tolist()),
    dict(name="adaptive_pw_and_near", kind="adaptive", norder=8, ipoly=0, iperiod=1, tree_eps=1e-6, maxlev=6,
         delta=1e-4, eps=1e-6, gauss=gauss(2, 6, 0.01, 0.05, normal=True, logw=True).tolist()),
    dict(name="adaptive_free_space", kind="adaptive", norder=8, ipoly=1, iperiod=0, tree_eps=1e-6, maxlev=6,
         delta=1e-4, eps=1e-9, gauss=gauss(2, 6, 0.01, 0.05, normal=True, logw=True).tolist()),
]


def main():
    out = {"generator": "tests/golden/make_golden.py", "cases": []}
    rng = np.random.default_rng(2024)
    for c in CASES:
        g = np.array(c["gauss"])
        if c["kind"] == "uniform":
            t = hb.build_uniform(c["level"], g, norder=c["norder"], ipoly=c["ipoly"], iperiod=c["iperiod"])
        else:
            t = hb.build_adaptive(g, norder=c["norder"], ipoly=c["ipoly"], iperiod=c["iperiod"], eps=c["tree_eps"],
                                  maxlev=c["maxlev"])
        if c.get("density") == "fourier22":
            xy = t.grid_points()
            t.fvals = np.sin(4 * np.pi * xy[..., 0]) * np.cos(4 * np.pi * xy[..., 1])
        q = quad.direct_pot(t, t.fvals, c["delta"]).reshape(t.nboxes, -1)
        lv = t.leaves()
        pick = rng.choice(len(lv) * t.npbox, size=min(256, len(lv) * t.npbox), replace=False)
        idx = np.stack([lv[pick // t.npbox], pick % t.npbox], 1)
        c = dict(c)
        c["nboxes"] = int(t.nboxes)
        c["sample_idx"] = idx.tolist()
        c["sample_pot"] = q[idx[:, 0], idx[:, 1]].tolist()
        out["cases"].append(c)
        print(c["name"], t.nboxes, "boxes", len(lv), "leaves")
    (Path(__file__).parent / "golden.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main()
