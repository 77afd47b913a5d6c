"""CPU tests of the C-ABI boundary: libykb.so loads, exports every symbol
include/ykb.h declares, builds the reference's geometry bit-exactly, and
rejects bad input with status codes (never aborting)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from fdk_cuda_impl_b200 import _lib as L
from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter, VolumeGrid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            names += re.findall(r"YKB_API\s+[\w\s\*]+?\b(ykb_\w+)\s*\(", text)
    return sorted(set(names))


def test_exports_every_declared_symbol(ykb_lib):
    names = declared_symbols()
    assert "ykb_fdk_execute" in names and "ykb_joseph_bp" in names
    for n in names:
        assert hasattr(ykb_lib, n), n
    # the Python binding table covers the same set
    assert set(names) <= set(L.SIGNATURES)


def test_version_and_scan_range(ykb_lib):
    assert ykb_lib.ykb_version() >= 100
    assert np.isclose(ykb_lib.ykb_regular_scan_range(180, 360), np.pi, rtol=1e-6)


@pytest.mark.parametrize("kw", [
    {},
    dict(start_angle_rad=0.3, rotation_direction=-1),
    dict(source_offset_mm=(0.5, -0.2, 0.1), offset_unv_mm=(1.2, 0.3, -0.7)),
    dict(tilt_rad=(0.14, 0.087, -0.07), z_mm=2.5),
])
def test_builder_bit_identical_to_oracle(ykb_lib, oracle, kw):
    sc = CircularScan(97, 90, 440.0, 770.0, 191, 97, 0.8, 0.6, **kw)
    a = sc.views()
    b = oracle.build_circular_flat(97, 90, 440.0, 770.0, 191, 97, 0.8, 0.6,
                                   start_angle=kw.get("start_angle_rad", 0.0),
                                   direction=kw.get("rotation_direction", 1),
                                   z=kw.get("z_mm", 0.0),
                                   source_offset=kw.get("source_offset_mm", (0, 0, 0)),
                                   offset_unv=kw.get("offset_unv_mm", (0, 0, 0)),
                                   tilt=kw.get("tilt_rad", (0, 0, 0)))
    assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("bad", [dict(sdd_mm=400.0), dict(views_per_turn=1),
                                 dict(rotation_direction=2), dict(channels=0),
                                 dict(channel_size_mm=0.0)])
def test_builder_rejects_invalid(ykb_lib, bad):
    base = dict(total_views=8, views_per_turn=8, sid_mm=500.0, sdd_mm=1000.0, channels=16,
                rows=8, channel_size_mm=1.0, row_size_mm=1.0)
    base.update(bad)
    with pytest.raises(L.YkbError) as e:
        CircularScan(**base).views()
    assert e.value.code == L.ERR_INVALID_GEOMETRY
    assert ykb_lib.ykb_last_error()


def test_builder_capacity_checked(ykb_lib):
    spec = CircularScan(8, 8, 500.0, 1000.0, 16, 8, 1.0, 1.0).spec()
    out = np.zeros(4, dtype=L.VIEW_DTYPE)
    assert ykb_lib.ykb_build_circular_flat(C.byref(spec), L.views_ptr(out), 4) == L.ERR_INVALID_BUFFER


def _plan(ykb_lib, views, nu=16, nv=8, grid=None, filt=None, precision=0, device=0):
    grid = grid or VolumeGrid.cube(8, 1.0)
    filt = filt or RampFilter()
    vs, fs = grid.struct(), filt.struct()
    h = C.c_void_p()
    rc = ykb_lib.ykb_fdk_plan_create(L.views_ptr(views) if views is not None else None,
                                     0 if views is None else len(views), nu, nv, 6.2831853,
                                     C.byref(vs), C.byref(fs), precision, device, C.byref(h))
    return rc, h


def test_plan_argument_validation_without_gpu(ykb_lib):
    views = CircularScan(8, 8, 500.0, 1000.0, 16, 8, 1.0, 1.0).views()
    assert _plan(ykb_lib, None)[0] == L.ERR_INVALID_CONFIG
    assert _plan(ykb_lib, views, grid=VolumeGrid(0, 8, 8))[0] == L.ERR_INVALID_CONFIG
    assert _plan(ykb_lib, views, filt=RampFilter(cutoff=0.7))[0] == L.ERR_INVALID_CONFIG
    assert _plan(ykb_lib, views, filt=RampFilter(type=12))[0] == L.ERR_INVALID_CONFIG
    assert _plan(ykb_lib, views, precision=5)[0] == L.ERR_INVALID_CONFIG
    vs, fs = VolumeGrid.cube(8, 1.0).struct(), RampFilter().struct()
    assert ykb_lib.ykb_fdk_plan_create(L.views_ptr(views), 8, 16, 8, 6.28, C.byref(vs),
                                       C.byref(fs), 0, 0, None) == L.ERR_INVALID_BUFFER
    # null plans are rejected, destroy(NULL) is a no-op
    assert ykb_lib.ykb_fdk_execute(None, None, 0, 0, 1, None, 1, None) == L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_joseph_fp(None, None, None, 0, None) == L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_fdk_plan_destroy(None) == L.OK


def test_no_device_reports_cuda_error(ykb_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    views = CircularScan(8, 8, 500.0, 1000.0, 16, 8, 1.0, 1.0).views()
    rc, _ = _plan(ykb_lib, views)
    assert rc in (L.ERR_CUDA, L.ERR_INVALID_CONFIG)
    assert ykb_lib.ykb_last_error()


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "fdk_cuda_impl_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cpp", ".cu", ".hpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.lower().replace("oracles", ""), f


def test_operator_and_solver_entry_points_validate_arguments(ykb_lib):
    # null plans and contexts are status codes, never a crash; the release
    # functions accept NULL
    assert ykb_lib.ykb_operator_apply(None, L.TASK_FP_JOSEPH, None, None, 0, None) == \
        L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_joseph_check(None, None) == L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_fdk_execute_host_out(None, None, 0, 0, 1, None, None, 1, None) == \
        L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_iter_create(0, None) == L.ERR_INVALID_BUFFER
    assert ykb_lib.ykb_iter_destroy(None) == L.OK
    assert ykb_lib.ykb_dot_f64(None, None, None, 0, None, None) == L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_cgls_update_xr(None, None, None, None, None, 0, None, None, 0, None) == \
        L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_cgls_update_p(None, None, None, None, None, 0, None) == \
        L.ERR_INVALID_CONFIG
    assert ykb_lib.ykb_joseph_plan_destroy(None) == L.OK


def test_solver_context_without_gpu(ykb_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert ykb_lib.ykb_iter_create(0, C.byref(h)) in (L.ERR_CUDA, L.ERR_INVALID_CONFIG)
    assert not h.value
    assert ykb_lib.ykb_last_error()
