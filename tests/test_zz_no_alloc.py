"""The no-allocation entry point (hrm_collatz_run_device_noalloc) against the regular one.

This entry point is for callers that cannot call cudaMalloc when they run a program (a
plug-in host that only hands out buffers registered ahead of time, or a service that forbids
allocation after start-up): it runs the runtime over a scratch area compiled into libhrm.so.
Its results must equal those of hrm_collatz_run_device (AsyncProgram, variant 0) bit for bit,
including on a second call in a row, which reuses the scratch area left by the first.
This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest


def _run(hrm, fn, start, count, out, **cfg_kw):
    cfg = hrm.make_config("async", **cfg_kw)
    res = hrm.RunResult()
    rc = fn(start, count, ctypes.c_void_p(out.data_ptr()), ctypes.byref(cfg), ctypes.byref(res))
    return rc, res.as_dict()


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_point_two_calls(hrm):
    import torch

    L = hrm.lib()
    f = L.hrm_collatz_run_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.POINTER(hrm.RunConfig),
                  ctypes.POINTER(hrm.RunResult)]
    for start, count in [(1, 1 << 18), (77777, 100003)]:
        out_na = torch.full((count,), -1, dtype=torch.int32, device="cuda")
        out_ref = torch.full((count,), -2, dtype=torch.int32, device="cuda")
        rc, res_na = _run(hrm, f, start, count, out_na)
        assert rc == hrm.HRM_OK, L.hrm_last_error().decode()
        rc, res_ref = _run(hrm, L.hrm_collatz_run_device, start, count, out_ref)
        assert rc == hrm.HRM_OK, L.hrm_last_error().decode()
        torch.cuda.synchronize()
        a = out_na.cpu().numpy().view(np.uint32)
        b = out_ref.cpu().numpy().view(np.uint32)
        assert np.array_equal(a, b)
        assert res_na["evals"] == res_ref["evals"]
        assert res_na["flags"] & hrm.FLAG_COMPLETION
