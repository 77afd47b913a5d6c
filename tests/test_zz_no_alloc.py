"""The allocation-free filter entry point (ykb_fdk_filter_static), called
through the C-ABI.

It serves callers that cannot call cudaMalloc (an application whose memory
pool owns the GPU, a real-time loop that forbids allocation after start-up);
its scratch is one fixed device array inside libykb.so.  The test runs two
calls in a row (the array keeps the previous call's contents) with different
view counts and dtypes, and checks each against the FP64 oracle's filter
stage with the filter-stage tolerance (5e-6 relative) and against the
plan-based ykb_fdk_filter on the same inputs; repeating both calls leaves
the device's free memory (cudaMemGetInfo) unchanged and the outputs equal.
This file is collected last so a failure here comes after every other test
has run."""
import ctypes as C

import numpy as np
import pytest

from tests import cases as K

pytestmark = pytest.mark.gpu

FILTER_TOL = 5e-6


def _static_filter(lib, L, views, nu, nv, scan_range, filt, proj, out):
    import torch
    fs = filt.struct()
    code = 1 if proj.dtype == torch.bfloat16 else 0
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.ykb_fdk_filter_static(L.views_ptr(views), len(views), nu, nv, scan_range,
                                     C.byref(fs), C.c_void_p(proj.data_ptr()), code,
                                     C.c_void_p(out.data_ptr()), stream)


def test_static_filter_matches_oracle_and_allocates_nothing(cuda_device, oracle):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.projectors import FdkPlan
    lib = L.load()
    case = K.c1_small()
    views = case.scan.views()
    nu, nv = case.scan.channels, case.scan.rows
    host = K.projections(oracle, case, views)
    p = torch.from_numpy(host).cuda()
    of = K.oracle_filter(oracle, case.filt)
    # second call: a different view subset, BF16 input, over the same scratch
    sub = np.ascontiguousarray(views[10:33])
    pb = p[10:33].to(torch.bfloat16).contiguous()
    out1 = torch.empty(p.shape, dtype=torch.float32, device="cuda")
    out2 = torch.empty(pb.shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    L.check(_static_filter(lib, L, views, nu, nv, case.scan.scan_range, case.filt, p, out1))
    L.check(_static_filter(lib, L, sub, nu, nv, case.scan.scan_range, case.filt, pb, out2))
    torch.cuda.synchronize()
    # once the library's kernels are loaded (lazily, by the first calls),
    # further calls leave the device's free memory unchanged
    first1, first2 = out1.clone(), out2.clone()
    free_before, _ = torch.cuda.mem_get_info()
    L.check(_static_filter(lib, L, views, nu, nv, case.scan.scan_range, case.filt, p, out1))
    L.check(_static_filter(lib, L, sub, nu, nv, case.scan.scan_range, case.filt, pb, out2))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert torch.equal(out1, first1) and torch.equal(out2, first2)

    ref1 = oracle.fdk_filter(views, nu, nv, case.scan.scan_range, of, host)
    assert K.rel_rmse(out1.cpu().numpy(), ref1) <= FILTER_TOL
    ref2 = oracle.fdk_filter(sub, nu, nv, case.scan.scan_range, of,
                             pb.float().cpu().numpy())
    assert K.rel_rmse(out2.cpu().numpy(), ref2) <= FILTER_TOL
    # the same arithmetic as the plan path's filter stage
    plan = FdkPlan(views, nu, nv, case.scan.scan_range, case.grid, case.filt)
    assert K.rel_rmse(out1.cpu().numpy(), plan.filter(p).cpu().numpy()) <= FILTER_TOL
    plan.close()


def test_static_filter_rejects_oversize_and_short_scans(cuda_device):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter
    lib = L.load()
    dummy = torch.zeros(16, device="cuda")
    fs = RampFilter().struct()
    scan = CircularScan(2, 2, 500.0, 1000.0, 8200, 4, 0.1, 0.1)
    views = scan.views()
    rc = lib.ykb_fdk_filter_static(L.views_ptr(views), 2, 8200, 4, scan.scan_range, C.byref(fs),
                                   C.c_void_p(dummy.data_ptr()), 0, C.c_void_p(dummy.data_ptr()),
                                   None)
    assert rc == L.ERR_INVALID_CONFIG
    assert b"8192" in lib.ykb_last_error()
    # 2816 x 2816 floats (31.7 MB) exceed the 30,867,456 rows bytes
    scan = CircularScan(2, 2, 500.0, 1000.0, 2816, 2816, 0.1, 0.1)
    views = scan.views()
    rc = lib.ykb_fdk_filter_static(L.views_ptr(views), 2, 2816, 2816, scan.scan_range,
                                   C.byref(fs), C.c_void_p(dummy.data_ptr()), 0,
                                   C.c_void_p(dummy.data_ptr()), None)
    assert rc == L.ERR_INVALID_CONFIG
    assert b"30867456" in lib.ykb_last_error()
    # a 240-degree scan needs Parker weights, which only a plan applies
    scan = CircularScan(240, 360, 500.0, 1000.0, 96, 64, 1.6, 1.6)
    views = scan.views()
    rc = lib.ykb_fdk_filter_static(L.views_ptr(views), 240, 96, 64, scan.scan_range, C.byref(fs),
                                   C.c_void_p(dummy.data_ptr()), 0, C.c_void_p(dummy.data_ptr()),
                                   None)
    assert rc == L.ERR_INVALID_CONFIG
    assert b"Parker" in lib.ykb_last_error()
