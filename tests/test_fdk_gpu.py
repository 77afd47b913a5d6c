"""GPU parity tests of the FDK path (through the C-ABI) against the FP64 oracle.

Tolerances: FP32 plans rel RMSE <= 1e-5 against the FP64 oracle (the FP32
target); BF16 plans rel RMSE <= 1e-3; stage outputs as stated per test.
"""
import numpy as np
import pytest

from tests import cases as K

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5
BF16_TOL = 1e-3


def _run_case(oracle, case, precision="fp32", proj_dtype="f32", ph=None):
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    views = case.scan.views()
    p = K.projections(oracle, case, views, ph)
    if proj_dtype == "bf16":
        pt = torch.from_numpy(p).to(torch.bfloat16)
        p = pt.float().numpy()
        dev_p = pt.cuda()
    else:
        dev_p = torch.from_numpy(p).cuda()
    plan = FdkPlan(views, case.scan.channels, case.scan.rows, case.scan.scan_range, case.grid,
                   case.filt, precision=precision)
    out = plan.execute(dev_p).cpu().numpy()
    plan.check()  # no device-side timeout or footprint error
    ref = oracle.fdk(views, case.scan.channels, case.scan.rows, case.scan.scan_range,
                     K.oracle_volume(oracle, case.grid), K.oracle_filter(oracle, case.filt), p)
    return out, ref, plan, views, p


def test_fdk_small_fp32(oracle, cuda_device):
    out, ref, *_ = _run_case(oracle, K.c1_small())
    assert np.isfinite(out).all()
    assert K.rel_rmse(out, ref) <= FP32_TOL


def test_fdk_c1_full_fp32(oracle, cuda_device):
    # 128^3 @ 0.5 mm, 180 views, 192x128 @ 0.8 mm, 500/1000 mm, Ram-Lak
    out, ref, *_ = _run_case(oracle, K.c1())
    assert K.rel_rmse(out, ref) <= FP32_TOL


def test_fdk_tilted_odd_sizes(oracle, cuda_device):
    # detector tilt + offsets + source offset + off-centre anisotropic grid:
    # exercises the general (non-axial) backprojection path
    out, ref, *_ = _run_case(oracle, K.odd_case())
    assert K.rel_rmse(out, ref) <= FP32_TOL


@pytest.mark.parametrize("kind", ["none", "shepplogan", "cosine", "hamming", "blackman",
                                  "butterworth", "kaiser", "tukey"])
def test_fdk_windows(oracle, cuda_device, kind):
    case = K.c1_small()
    case.filt = K.RampFilter.named(kind, cutoff=0.45)
    out, ref, *_ = _run_case(oracle, case)
    assert K.rel_rmse(out, ref) <= FP32_TOL


@pytest.mark.parametrize("path", ["tensor", "simt"])
def test_fdk_filter_stage(oracle, cuda_device, monkeypatch, path):
    # FP32 plans filter on the tensor cores with three BF16 parts per operand
    # (six products) or, with YKB_FDK_FILTER=simt, with FP32 FMAs
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    if path == "simt":
        monkeypatch.setenv("YKB_FDK_FILTER", "simt")
    case = K.c1_small()
    views = case.scan.views()
    p = K.projections(oracle, case, views)
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
    got = plan.filter(torch.from_numpy(p).cuda()).cpu().numpy()
    ref = oracle.fdk_filter(views, 96, 64, case.scan.scan_range,
                            K.oracle_filter(oracle, case.filt), p)
    # the ramp output cancels large lags of both signs: an FP32 sum over nu
    # lags keeps a few 1e-6 relative; the volume target (1e-5) is end to end
    assert K.rel_rmse(got, ref) <= 5e-6


def test_fdk_backproject_stage(oracle, cuda_device):
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    f = oracle.normal((60, 64, 96), 21)
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
    got = plan.backproject(torch.from_numpy(f).cuda()).cpu().numpy()
    plan.check()
    ref = oracle.fdk_backproject(views, 96, 64, case.scan.scan_range,
                                 K.oracle_volume(oracle, case.grid), f.astype(np.float64))
    assert K.rel_rmse(got, ref) <= FP32_TOL


def test_fdk_streaming_batches(oracle, cuda_device):
    # fdk/batch-consistency (Yktest/test_pipeline_smoke.cpp:2077-2122): a run
    # split into contiguous batches equals the full run (pin: max diff < 1e-4)
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views)).cuda()
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
    full = plan.execute(p).clone()
    vol = torch.full(case.grid.shape, 123.0, device="cuda")
    plan.execute(p[0:5], vol, view_offset=0, clear=True)
    plan.execute(p[5:23], vol, view_offset=5, clear=False)
    plan.execute(p[23:], vol, view_offset=23, clear=False)
    plan.check()
    diff = (vol - full).abs().max().item()
    assert diff < 1e-4
    assert K.rel_rmse(vol.cpu().numpy(), full.cpu().numpy()) < 1e-6


def test_fdk_bf16_form(oracle, cuda_device):
    out, ref, *_ = _run_case(oracle, K.c1_small(), precision="bf16")
    assert K.rel_rmse(out, ref) <= BF16_TOL


def test_fdk_bf16_projection_input(oracle, cuda_device):
    out, ref, *_ = _run_case(oracle, K.c1_small(), proj_dtype="bf16")
    assert K.rel_rmse(out, ref) <= FP32_TOL


def test_fdk_extreme_detector_offset(oracle, cuda_device):
    # principal point far outside the detector: the padded FFT row drops
    # samples; the Toeplitz form must drop exactly the same ones
    case = K.c1_small()
    case.scan.offset_unv_mm = (135.0, 0.0, 5.0)
    out, ref, *_ = _run_case(oracle, case)
    d = oracle.fdk_derived(case.scan.views(), 96, 64, case.scan.scan_range)
    N = 256
    assert ((d[:, 10] < 0) | (d[:, 10] + 96 > N)).any()  # masks are active
    assert K.rel_rmse(out, ref) <= FP32_TOL


def test_fdk_noisy_short_views(oracle, cuda_device):
    case = K.c1_small()
    case.noise_i0 = 5e4
    out, ref, *_ = _run_case(oracle, case)
    assert K.rel_rmse(out, ref) <= FP32_TOL


def test_fdk_errors_are_status_codes(cuda_device, oracle):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    plan = FdkPlan(case.scan.views(), 96, 64, case.scan.scan_range, case.grid, case.filt)
    p = torch.zeros((10, 64, 96), device="cuda")
    with pytest.raises(L.YkbError) as e:
        plan.execute(p, view_offset=55)
    assert e.value.code == L.ERR_INVALID_CONFIG
    # the context stays usable
    assert torch.isfinite(plan.execute(p, view_offset=50)).all()


def test_fdk_backproject_stage_unaligned_pitch(oracle, cuda_device):
    # nu not a multiple of 4: the stage entry cannot use a TMA tensor map on
    # the caller's buffer and takes the global-load kernel
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.odd_case()
    views = case.scan.views()
    nu, nv = case.scan.channels, case.scan.rows
    f = oracle.normal((len(views), nv, nu), 31)
    plan = FdkPlan(views, nu, nv, case.scan.scan_range, case.grid, case.filt)
    got = plan.backproject(torch.from_numpy(f).cuda()).cpu().numpy()
    plan.check()
    ref = oracle.fdk_backproject(views, nu, nv, case.scan.scan_range,
                                 K.oracle_volume(oracle, case.grid), f.astype(np.float64))
    assert K.rel_rmse(got, ref) <= FP32_TOL


def test_fdk_tma_matches_global_path(oracle, cuda_device):
    # the three backprojection paths -- TMA-staged tap pairs (default),
    # TMA-staged plain rows, global loads -- give the same volume: the same
    # weights applied in the same order, up to FP32 rounding of the lerps
    import os
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views)).cuda()
    out = {}
    for path in ("pairs", "rows", "global"):
        if path == "pairs":
            os.environ.pop("YKB_FDK_BP_PATH", None)
        else:
            os.environ["YKB_FDK_BP_PATH"] = path
        try:
            plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
        finally:
            os.environ.pop("YKB_FDK_BP_PATH", None)
        out[path] = plan.execute(p).cpu().numpy()
        filtered = plan.filter(p)
        # the stage entry with a buffer 4 bytes off a 16-byte boundary
        flat = torch.empty(filtered.numel() + 1, device="cuda")
        shifted = flat[1:].view(filtered.shape)
        shifted.copy_(filtered)
        assert shifted.data_ptr() % 16 != 0
        staged = plan.backproject(shifted).cpu().numpy()
        plan.check()
        assert K.rel_rmse(staged, out[path]) < 1e-6, path
        plan.close()
    assert K.rel_rmse(out["rows"], out["pairs"]) < 1e-6
    assert K.rel_rmse(out["global"], out["pairs"]) < 1e-6


@pytest.mark.parametrize("path", ["tensor", "simt"])
@pytest.mark.parametrize("nu", [768, 1536])
def test_fdk_filter_stage_wide(oracle, cuda_device, monkeypatch, nu, path):
    # the FP32 Toeplitz filter at the detector widths of the 512^3 and 1024^3
    # workloads
    import torch
    if path == "simt":
        monkeypatch.setenv("YKB_FDK_FILTER", "simt")
    from fdk_cuda_impl_b200.geometry import CircularScan
    from fdk_cuda_impl_b200.projectors import FdkPlan
    scan = CircularScan(3, 3, 500.0, 1000.0, nu, 6, 0.4, 0.4)
    v = scan.views()
    case = K.c1_small()
    p = oracle.uniform((3, 6, nu), 0.0, 2.0, 50 + nu)
    plan = FdkPlan(v, nu, 6, scan.scan_range, case.grid, case.filt)
    got = plan.filter(torch.from_numpy(p).cuda()).cpu().numpy()
    plan.check()
    ref = oracle.fdk_filter(v, nu, 6, scan.scan_range, K.oracle_filter(oracle, case.filt), p)
    # FP32 sums over nu lags that largely cancel: the error grows with the
    # row (measured 5.8e-6 on the tensor cores at nu = 1536)
    assert K.rel_rmse(got, ref) <= 5e-6 * max(1.0, nu / 768)


@pytest.mark.parametrize("kind,cutoff", [("ramlak", 0.5), ("hamming", 0.5), ("ramlak", 0.3),
                                         ("tukey", 0.45)])
def test_tc_filter_near_band_matches_full_band(oracle, cuda_device, monkeypatch, kind, cutoff):
    # FP32 plans run their three 2^-16 products only over the K chunks near
    # each output tile when the taps beyond are small (1/d^2 tails); a slow
    # tail (a sharp cut-off below Nyquist) keeps more chunks.  Smooth rows:
    # the ramp output cancels most of the lag sum
    import torch
    from fdk_cuda_impl_b200.geometry import CircularScan
    from fdk_cuda_impl_b200.projectors import FdkPlan
    nu, nv = 1536, 6
    scan = CircularScan(3, 3, 500.0, 1000.0, nu, nv, 0.4, 0.4)
    v = scan.views()
    case = K.c1_small()
    filt = K.RampFilter.named(kind, cutoff=cutoff)
    u = (np.arange(nu) - nu / 2 + 0.3) / (0.35 * nu)
    disc = 100.0 * np.sqrt(np.clip(1.0 - u * u, 0.0, None))
    p = (disc[None, None, :] + oracle.uniform((3, nv, nu), -0.5, 0.5, 61)).astype(np.float32)
    out = {}
    for near in ("auto", "1000"):
        if near == "auto":
            monkeypatch.delenv("YKB_FDK_FILTER_NEAR", raising=False)
        else:
            monkeypatch.setenv("YKB_FDK_FILTER_NEAR", near)
        plan = FdkPlan(v, nu, nv, scan.scan_range, case.grid, filt)
        out[near] = plan.filter(torch.from_numpy(p).cuda()).cpu().numpy()
        plan.check()
        plan.close()
    ref = oracle.fdk_filter(v, nu, nv, scan.scan_range, K.oracle_filter(oracle, filt), p)
    full, near = K.rel_rmse(out["1000"], ref), K.rel_rmse(out["auto"], ref)
    # FP32 sums over 1536 lags (the full band measured 1.0e-5 for Hamming)
    assert full <= 2e-5
    assert near <= 1.1 * full


@pytest.mark.parametrize("nu,nv,views", [(96, 64, 12), (53, 41, 7), (192, 24, 5), (384, 8, 3),
                                         (768, 8, 2), (1536, 6, 2)])
def test_tc_filter_stage(oracle, cuda_device, nu, nv, views):
    # tcgen05 BF16 Toeplitz filter with hi/lo split against the FP64 filter:
    # the three-product split keeps about 16 mantissa bits
    import torch
    from fdk_cuda_impl_b200.geometry import CircularScan
    from fdk_cuda_impl_b200.projectors import FdkPlan
    scan = CircularScan(views, views, 500.0, 1000.0, nu, nv, 1.0, 1.0)
    v = scan.views()
    case = K.c1_small()
    p = oracle.uniform((views, nv, nu), 0.0, 2.0, 40 + nu)
    plan = FdkPlan(v, nu, nv, scan.scan_range, case.grid, case.filt, precision="bf16")
    got = plan.filter(torch.from_numpy(p).cuda()).cpu().numpy()
    plan.check()
    ref = oracle.fdk_filter(v, nu, nv, scan.scan_range, K.oracle_filter(oracle, case.filt), p)
    assert got.dtype == np.float32
    assert K.rel_rmse(got, ref) <= 1e-4


def test_bf16_form_c1(oracle, cuda_device):
    # BF16 projections in, tensor-core filter: end-to-end bound 1e-3
    out, ref, *_ = _run_case(oracle, K.c1(), precision="bf16", proj_dtype="bf16")
    assert K.rel_rmse(out, ref) <= BF16_TOL


@pytest.mark.parametrize("precision,tol", [("fp32", FP32_TOL), ("bf16", BF16_TOL)])
@pytest.mark.parametrize("tilted", [False, True])
def test_fdk_filter_column_tiles(oracle, cuda_device, precision, tol, tilted):
    # nu = 300 runs the tensor-core filter in five 64-column tiles; the tap
    # pair across each tile edge is written in halves by two CTAs.  The
    # 37-row detector truncates the volume's projection, so the first and
    # last rows are sampled too.
    from fdk_cuda_impl_b200.geometry import CircularScan, VolumeGrid
    kw = dict(tilt_rad=(0.01, -0.015, 0.02), offset_unv_mm=(2.1, 0.0, -1.3)) if tilted else {}
    case = K.c1_small()
    case.scan = CircularScan(40, 40, 500.0, 1000.0, 300, 37, 0.5, 1.7, **kw)
    case.grid = VolumeGrid(64, 64, 40, (1.0, 1.0, 1.0))
    out, ref, plan, *_ = _run_case(oracle, case, precision=precision)
    assert np.isfinite(out).all()
    assert K.rel_rmse(out, ref) <= tol
    plan.close()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_fdk_execute_host_matches_device(oracle, cuda_device, pinned, precision):
    # host-input streaming FDK (batched copies overlapping the kernels) gives
    # the device-input result; the batches only reorder the view sums
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views))
    if precision == "bf16":
        p = p.to(torch.bfloat16)
    host = p.pin_memory() if pinned else p.clone()
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt, precision)
    dev = plan.execute(p.cuda()).cpu().numpy()
    streamed = plan.execute_host(host)
    torch.cuda.current_stream().synchronize()
    plan.check()
    assert K.rel_rmse(streamed.cpu().numpy(), dev) < 1e-6
    # accumulate: two calls over halves equal one call
    vol = plan.execute_host(host[:30].contiguous())
    plan.execute_host(host[30:].contiguous(), vol, view_offset=30, clear=False)
    torch.cuda.current_stream().synchronize()
    assert K.rel_rmse(vol.cpu().numpy(), dev) < 1e-6
    plan.close()


@pytest.mark.parametrize("nz", [48, 100])
def test_fdk_execute_host_out(oracle, cuda_device, nz):
    # host projections in, host volume out: the last batch runs in z slabs of
    # whole 48-slice z tiles whose downloads overlap the next slab (nz = 48:
    # one slab; nz = 100: slabs of 48, 48 and 4 slices)
    import torch
    from fdk_cuda_impl_b200.geometry import VolumeGrid
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    case.grid = VolumeGrid(64, 64, nz, (1.0, 1.0, 48.0 / nz))
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views))
    plan = FdkPlan(views, 96, 64, case.scan.scan_range, case.grid, case.filt)
    dev = plan.execute(p.cuda()).cpu().numpy()
    host = p.pin_memory()
    out = torch.empty(case.grid.shape, dtype=torch.float32).pin_memory()
    out.fill_(float("nan"))
    for _ in range(2):  # a second call reuses the staging and events
        vol = plan.execute_host(host, host_out=out)
        torch.cuda.current_stream().synchronize()
        plan.check()
        assert K.rel_rmse(out.numpy(), dev) < 1e-6
        assert torch.equal(out, vol.cpu())
    plan.close()


def _short_scan_case(start=0.3, direction=-1):
    from fdk_cuda_impl_b200.geometry import CircularScan
    case = K.c1_small()
    # 40 views of a 60-view turn: 240 degrees >= 180 + 2 x 4.4 degrees of fan
    case.scan = CircularScan(40, 60, 500.0, 1000.0, 96, 64, 1.6, 1.6, start_angle_rad=start,
                             rotation_direction=direction)
    return case


@pytest.mark.parametrize("precision,tol", [("fp32", FP32_TOL), ("bf16", BF16_TOL)])
@pytest.mark.parametrize("direction", [1, -1])
def test_fdk_parker_short_scan(oracle, cuda_device, precision, tol, direction):
    # short-scan FDK with Parker weights (Auto on a 240-degree scan) against
    # the oracle's restatement of the reference weights
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = _short_scan_case(direction=direction)
    sc = case.scan
    views = sc.views()
    p = K.projections(oracle, case, views)
    plan = FdkPlan(views, 96, 64, sc.scan_range, case.grid, case.filt, precision, parker="auto",
                   start_angle_rad=sc.start_angle_rad, rotation_direction=direction)
    out = plan.execute(torch.from_numpy(p).cuda()).cpu().numpy()
    plan.check()
    w = oracle.parker_weights(views, 96, 64, sc.scan_range, sc.start_angle_rad, direction)
    ref = oracle.fdk_weighted(views, 96, 64, sc.scan_range, K.oracle_volume(oracle, case.grid),
                              K.oracle_filter(oracle, case.filt), p, w)
    assert K.rel_rmse(out, ref) <= tol
    plan.close()


def test_fdk_parker_modes(oracle, cuda_device):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = _short_scan_case()
    sc = case.scan
    views = sc.views()
    p = K.projections(oracle, case, views)
    # Disabled: plain FDK of the short scan
    plan = FdkPlan(views, 96, 64, sc.scan_range, case.grid, case.filt, parker="disabled",
                   start_angle_rad=sc.start_angle_rad, rotation_direction=-1)
    out = plan.execute(torch.from_numpy(p).cuda()).cpu().numpy()
    ref = oracle.fdk(views, 96, 64, sc.scan_range, K.oracle_volume(oracle, case.grid),
                     K.oracle_filter(oracle, case.filt), p)
    assert K.rel_rmse(out, ref) <= FP32_TOL
    plan.close()
    # Enabled on a full turn, or on a scan shorter than pi + 2 fan: invalid geometry
    full = K.c1_small()
    with pytest.raises(L.YkbError) as e:
        FdkPlan(full.scan.views(), 96, 64, full.scan.scan_range, full.grid, parker="enabled")
    assert e.value.code == L.ERR_INVALID_GEOMETRY
    from fdk_cuda_impl_b200.geometry import CircularScan
    half = CircularScan(30, 60, 500.0, 1000.0, 96, 64, 1.6, 1.6)
    with pytest.raises(L.YkbError) as e:
        FdkPlan(half.views(), 96, 64, half.scan_range, full.grid, parker="auto")
    assert e.value.code == L.ERR_INVALID_GEOMETRY
    # Auto on a full turn: no weights
    plan = FdkPlan(full.scan.views(), 96, 64, full.scan.scan_range, full.grid, parker="auto")
    plan.close()


@pytest.mark.parametrize("withheld", [0, 5, 59])
def test_pipeline_wait_timeout_is_reported_and_the_plan_recovers(oracle, cuda_device, withheld):
    # The TMA backprojection bounds every pipeline wait.  The test hook makes
    # the copy producer withhold one view and shortens the waits to 1 ms:
    # every CTA's consumers give up on that view, its producer gives up on
    # the stage they never release, drains the copies it issued and ends.
    # ykb_fdk_check reports the timeout; afterwards the same plan, with the
    # default limit restored, reproduces its earlier result bit for bit.
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views)).cuda()
    plan = FdkPlan(views, case.scan.channels, case.scan.rows, case.scan.scan_range, case.grid,
                   case.filt)
    expected = plan.execute(p).clone()
    plan.check()
    lib = L.load()
    L.check(lib.ykb_fdk_test_pipeline_wait(plan._h, 1_000_000, withheld))
    plan.execute(p)
    with pytest.raises(L.YkbError, match="pipeline wait timed out"):
        plan.check()
    L.check(lib.ykb_fdk_test_pipeline_wait(plan._h, 0, -1))
    again = plan.execute(p)
    plan.check()
    assert torch.equal(again, expected)
    plan.close()


def test_stage_timing_counts_launch_groups(oracle, cuda_device):
    # ykb_fdk_stage_timing records one event pair per filter and per
    # backprojection launch group; the tally restarts after each read
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan
    case = K.c1_small()
    views = case.scan.views()
    p = torch.from_numpy(K.projections(oracle, case, views)).cuda()
    plan = FdkPlan(views, case.scan.channels, case.scan.rows, case.scan.scan_range, case.grid,
                   case.filt)
    plan.stage_timing(True)
    for _ in range(3):
        plan.execute(p)
    t = plan.stage_times()
    assert t["filter_groups"] == 3 and t["backproject_groups"] == 3
    assert t["filter_ms"] > 0 and t["backproject_ms"] > 0
    assert plan.stage_times()["backproject_groups"] == 0
    plan.stage_timing(False)
    plan.execute(p)
    assert plan.stage_times()["filter_groups"] == 0
    plan.check()
    plan.close()
