"""The allocation-free filter entry point (ykb_fdk_filter_static), called
through the C-ABI, against the plan-based ykb_fdk_filter on the same inputs.

It serves callers that cannot call cudaMalloc; its scratch is one fixed
device array inside libykb.so.  The test runs two calls in a row (the array
keeps the previous call's contents) with different view counts and dtypes,
and compares with the tolerance of the filter-stage test (5e-6 relative,
here against the plan path, which computes the same arithmetic)."""
import ctypes as C

import numpy as np
import pytest

from tests import cases as K

pytestmark = pytest.mark.gpu


def _static_filter(lib, L, views, nu, nv, scan_range, filt, proj):
    import torch
    out = torch.empty(proj.shape, dtype=torch.float32, device=proj.device)
    fs = filt.struct()
    code = 1 if proj.dtype == torch.bfloat16 else 0
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.ykb_fdk_filter_static(L.views_ptr(views), len(views), nu, nv, scan_range,
                                   C.byref(fs), C.c_void_p(proj.data_ptr()), code,
                                   C.c_void_p(out.data_ptr()), stream)
    L.check(rc)
    return out


def test_static_filter_matches_plan_filter(cuda_device, oracle):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.projectors import FdkPlan
    lib = L.load()
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views)).cuda()
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
    expected = plan.filter(p)
    # first call: all 60 views
    got1 = _static_filter(lib, L, views, 96, 64, case.scan.scan_range, case.filt, p)
    torch.cuda.synchronize()
    assert K.rel_rmse(got1.cpu().numpy(), expected.cpu().numpy()) <= 5e-6
    # second call in a row: a different subset and bf16 input over the same scratch
    sub = np.ascontiguousarray(views[10:33])
    pb = p[10:33].to(torch.bfloat16).contiguous()
    got2 = _static_filter(lib, L, sub, 96, 64, case.scan.scan_range, case.filt, pb)
    plan2 = FdkPlan(sub, 96, 64, case.scan.scan_range, case.grid, case.filt)
    expected2 = plan2.filter(pb)
    torch.cuda.synchronize()
    assert K.rel_rmse(got2.cpu().numpy(), expected2.cpu().numpy()) <= 5e-6


def test_static_filter_rejects_oversize(cuda_device):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter
    lib = L.load()
    scan = CircularScan(2, 2, 500.0, 1000.0, 8200, 4, 0.1, 0.1)
    views = scan.views()
    dummy = torch.zeros(16, device="cuda")
    fs = RampFilter().struct()
    rc = lib.ykb_fdk_filter_static(L.views_ptr(views), 2, 8200, 4, scan.scan_range, C.byref(fs),
                                   C.c_void_p(dummy.data_ptr()), 0, C.c_void_p(dummy.data_ptr()),
                                   None)
    assert rc == L.ERR_INVALID_CONFIG
    assert b"8192" in lib.ykb_last_error()
