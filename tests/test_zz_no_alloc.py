"""bfgt_plan_execute_noalloc: the planned transform without any device
allocation, for callers that may not allocate while they step (a solver whose
memory manager owns the device, or a loop that cannot afford the stalls of
cudaMalloc/cudaFree).  Its plane-wave scratch lives in a static array inside
the library.  Checked through the C ABI
against bfgt_plan_execute on two calls in a row, with the tolerances of the
other GPU tests (FP64: 1e-11 relative L2; split precision: 1e-6)."""
import ctypes as C

import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from heat2d_per_box_b200 import _lib

pytestmark = pytest.mark.gpu


def _tree():
    rng = np.random.default_rng(12)
    g = hb.gauss_params(rng.uniform(-0.5, 0.5, (6, 2)), np.exp(rng.uniform(np.log(0.01), np.log(0.05), 6)),
                        rng.standard_normal(6))
    return hb.build_adaptive(g, norder=16, ipoly=0, iperiod=1, eps=1e-8, maxlev=5)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,tol", [(hb.BFGT_PREC_FP64, 1e-11), (hb.BFGT_PREC_SPLIT, 1e-6)])
def test_noalloc_matches_planned_execute(precision, tol):
    import torch
    t = _tree()
    plan = hb.Plan(t, 1e-4, 1e-6, precision=precision)
    L = _lib.lib()
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    ref = torch.zeros_like(f)
    plan.execute(f, ref)
    torch.cuda.synchronize()
    lv = t.leaves()
    r = ref.cpu().numpy().reshape(t.nboxes, -1)[lv]
    for _ in range(2):  # the static scratch keeps the previous call's contents
        out = torch.zeros_like(f)
        rc = L.bfgt_plan_execute_noalloc(plan._h, C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.bfgt_last_error().decode()
        torch.cuda.synchronize()
        plan.check()
        o = out.cpu().numpy().reshape(t.nboxes, -1)[lv]
        assert rel_l2(o, r) < tol
    plan.close()


def test_noalloc_rejects_plans_beyond_the_static_scratch():
    t = _tree()
    nd = 64
    plan = hb.Plan(t, 1e-4, 1e-6, nd=nd)
    L = _lib.lib()
    cap = C.c_size_t()
    assert L.bfgt_noalloc_scratch_bytes(C.byref(cap)) == 0
    assert plan.noalloc_need() > cap.value
    rc = L.bfgt_plan_execute_noalloc(plan._h, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 3  # BFGT_ERR_CAPACITY
    assert "static scratch" in L.bfgt_last_error().decode()
    plan.close()
