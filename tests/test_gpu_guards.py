"""The device-array entry points check where their arrays live before any
kernel runs: a host array (pageable or page-locked) handed to
bfgt_plan_execute, bfgt_plan_execute_pgh, bfgt_plan_execute_adjoint,
bfgt_plan_graph_capture or bfgt_batch_execute is refused with BFGT_ERR_ARG
(a kernel reading it would fault), and the plan stays usable."""
import ctypes as C

import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from heat2d_per_box_b200 import _lib

pytestmark = pytest.mark.gpu


def test_host_arrays_are_refused_by_device_entry_points(trees):
    import torch
    t = trees["ad_leg_per"]
    plan = hb.Plan(t, 1e-4, 1e-6)
    L = _lib.lib()
    f = torch.from_numpy(t.fvals.reshape(-1)).cuda()
    p = torch.zeros_like(f)
    host = np.zeros(f.numel())
    pinned = torch.zeros(f.numel(), dtype=torch.float64).pin_memory()
    for bad in (host.ctypes.data, pinned.data_ptr()):
        rc = L.bfgt_plan_execute(plan._h, C.c_void_p(f.data_ptr()), C.c_void_p(bad), None)
        assert rc == 1
        msg = L.bfgt_last_error()
        assert b"not device memory" in msg or b"not a CUDA allocation" in msg, msg
        rc = L.bfgt_plan_execute_pgh(plan._h, 2, C.c_void_p(f.data_ptr()), C.c_void_p(p.data_ptr()), C.c_void_p(bad),
                                     None, None)
        assert rc == 1
        rc = L.bfgt_plan_execute_adjoint(plan._h, C.c_void_p(bad), C.c_void_p(p.data_ptr()), None)
        assert rc == 1
        rc = L.bfgt_plan_graph_capture(plan._h, C.c_void_p(bad), C.c_void_p(p.data_ptr()), None)
        assert rc == 1
    batch = hb.Batch([plan])
    rc = L.bfgt_batch_execute(batch._h, C.c_void_p(host.ctypes.data), C.c_void_p(p.data_ptr()), None)
    assert rc == 1
    # the plan still works, and matches a fresh run
    plan.execute(f, p)
    plan.check()
    q = torch.zeros_like(f)
    batch.execute(f, q)
    batch.check()
    np.testing.assert_array_equal(p.cpu().numpy(), q.cpu().numpy())
    batch.close()
    plan.close()
