"""GPU tests of the Joseph projector pair: parity with the FP64 oracle,
the dot-product (adjoint) test in FP64, finite differences of 1/2||Ax-b||^2
through the autograd Function, and write modes."""
import numpy as np
import pytest

from tests import cases as K
from fdk_cuda_impl_b200.geometry import CircularScan, VolumeGrid

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5
ADJ_TOL = 1e-6


def _plan(case):
    from fdk_cuda_impl_b200.projectors import JosephPlan
    views = case.scan.views()
    return views, JosephPlan(views, case.scan.channels, case.scan.rows, case.grid)


def _z_axis_views(oracle):
    # views looking along z (source below the volume): main axis Z
    v = np.zeros(6, dtype=oracle.VIEW_DTYPE)
    for i in range(6):
        a = 2 * np.pi * i / 6
        v[i]["src"][:3] = [20 * np.cos(a), 20 * np.sin(a), -300.0]
        v[i]["detS"][:3] = [-31.5 * 1.2, -23.5 * 1.2, 250.0]
        v[i]["detU"][:3] = [1.2, 0, 0]
        v[i]["detV"][:3] = [0, 1.2, 0]
        v[i]["angle"][0] = a
    return v


def test_fp_matches_oracle(oracle, cuda_device):
    import torch
    case = K.c1_small()
    views, plan = _plan(case)
    x = K.phantom(oracle, case)
    got = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = oracle.joseph_fp(views, 96, 64, K.oracle_volume(oracle, case.grid), x)
    assert set(np.unique(oracle.joseph_main_axes(views, 96, 64))) == {0, 1}
    assert K.rel_rmse(got, ref) <= FP32_TOL


def test_bp_matches_oracle(oracle, cuda_device):
    import torch
    case = K.c1_small()
    views, plan = _plan(case)
    y = oracle.normal(plan.proj_shape, 3)
    got = plan.adjoint(torch.from_numpy(y).cuda()).cpu().numpy()
    ref = oracle.joseph_bp(views, 96, 64, K.oracle_volume(oracle, case.grid), y)
    assert K.rel_rmse(got, ref) <= FP32_TOL


def test_tilted_anisotropic_fp_bp(oracle, cuda_device):
    import torch
    case = K.odd_case()
    views, plan = _plan(case)
    vol = K.oracle_volume(oracle, case.grid)
    x = oracle.uniform(case.grid.shape, 0.0, 1.0, 8)
    y = oracle.normal(plan.proj_shape, 9)
    fp = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    bp = plan.adjoint(torch.from_numpy(y).cuda()).cpu().numpy()
    assert K.rel_rmse(fp, oracle.joseph_fp(views, case.scan.channels, case.scan.rows, vol, x)) <= FP32_TOL
    assert K.rel_rmse(bp, oracle.joseph_bp(views, case.scan.channels, case.scan.rows, vol, y)) <= FP32_TOL


def test_z_main_axis(oracle, cuda_device):
    import torch
    from fdk_cuda_impl_b200.projectors import JosephPlan
    views = _z_axis_views(oracle)
    grid = VolumeGrid(40, 30, 24, (1.0, 1.0, 1.5))
    assert (oracle.joseph_main_axes(views, 64, 48) == 2).all()
    plan = JosephPlan(views, 64, 48, grid)
    vol = K.oracle_volume(oracle, grid)
    x = oracle.uniform(grid.shape, 0.0, 1.0, 4)
    y = oracle.normal(plan.proj_shape, 5)
    fp = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    bp = plan.adjoint(torch.from_numpy(y).cuda()).cpu().numpy()
    assert K.rel_rmse(fp, oracle.joseph_fp(views, 64, 48, vol, x)) <= FP32_TOL
    assert K.rel_rmse(bp, oracle.joseph_bp(views, 64, 48, vol, y)) <= FP32_TOL


def _adjoint_error(plan, grid, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.rand(grid.shape, generator=g, device="cuda")
    y = torch.randn(plan.proj_shape, generator=g, device="cuda")
    ax = plan.forward(x)
    aty = plan.adjoint(y)
    lhs = (ax.double() * y.double()).sum().item()
    rhs = (x.double() * aty.double()).sum().item()
    return abs(lhs - rhs) / max(abs(lhs), abs(rhs))


def test_adjoint_small(cuda_device):
    case = K.c1_small()
    _, plan = _plan(case)
    assert _adjoint_error(plan, case.grid, 1) <= ADJ_TOL


def test_adjoint_c3_full(cuda_device):
    # 256^3, 360 views, 384x384 detector; x ~ U[0,1], y ~ N(0,1)
    from fdk_cuda_impl_b200.projectors import JosephPlan
    scan = CircularScan(360, 360, 500.0, 1000.0, 384, 384, 0.8, 0.8)
    grid = VolumeGrid.cube(256, 0.5)
    plan = JosephPlan(scan.views(), 384, 384, grid)
    assert _adjoint_error(plan, grid, 2) <= ADJ_TOL


def test_reference_adjoint_pin(oracle, cuda_device):
    # unit_test/test_operator_benchmarks.cpp:847-990 "representative" shape:
    # 96x96x64 @ 1 mm, 192x96 @ 0.8 mm, 180 views, SID/SDD 440/770, inputs
    # from std::mt19937 seeds 12345/54321 on U[-1,1]; the reference asserts
    # Joseph FP + BP_Joseph adjoint error < 5e-3 (its texture filter), here
    # the exact transpose must reach the FP64-level bound.
    import torch
    from fdk_cuda_impl_b200.projectors import JosephPlan
    scan = CircularScan(180, 180, 440.0, 770.0, 192, 96, 0.8, 0.8)
    grid = VolumeGrid(96, 96, 64, (1.0, 1.0, 1.0))
    plan = JosephPlan(scan.views(), 192, 96, grid)
    x = oracle.mt19937_uniform_pm1(96 * 96 * 64, 12345).reshape(grid.shape)
    y = oracle.mt19937_uniform_pm1(180 * 96 * 192, 54321).reshape(plan.proj_shape)
    ax = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy().astype(np.float64)
    aty = plan.adjoint(torch.from_numpy(y).cuda()).cpu().numpy().astype(np.float64)
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    err = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    assert err < 5e-3
    assert err <= ADJ_TOL


def test_finite_differences(cuda_device):
    # gradient of 1/2||Ax-b||^2 (FP64 reduction) at 64 random voxels, eps=1e-3
    import torch
    from fdk_cuda_impl_b200.autograd import project
    case = K.c1_small()
    _, plan = _plan(case)
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand(case.grid.shape, generator=g, device="cuda")
    b = torch.randn(plan.proj_shape, generator=g, device="cuda")
    xr = x.clone().requires_grad_(True)
    loss = 0.5 * ((project(xr, plan) - b).double() ** 2).sum()
    loss.backward()
    grad = xr.grad.double()
    idx = torch.randint(0, x.numel(), (64,), generator=g, device="cuda")
    eps = 1e-3

    def f(v):
        with torch.no_grad():
            return 0.5 * ((plan.forward(v) - b).double() ** 2).sum().item()

    errs = []
    for i in idx.tolist():
        xp = x.clone().view(-1); xp[i] += eps
        xm = x.clone().view(-1); xm[i] -= eps
        fd = (f(xp.view(x.shape)) - f(xm.view(x.shape))) / (2 * eps)
        an = grad.view(-1)[i].item()
        errs.append(abs(fd - an) / max(abs(an), 1e-3))
    assert max(errs) < 1e-2
    assert float(np.median(errs)) < 1e-3


def test_write_modes(cuda_device):
    import torch
    case = K.c1_small()
    _, plan = _plan(case)
    x = torch.rand(case.grid.shape, device="cuda")
    y = torch.randn(plan.proj_shape, device="cuda")
    p1 = plan.forward(x)
    p2 = torch.ones_like(p1)
    plan.forward(x, out=p2, accumulate=True)
    assert torch.allclose(p2, p1 + 1, atol=1e-4)
    v1 = plan.adjoint(y)
    v2 = torch.full_like(v1, 2.0)
    plan.adjoint(y, out=v2, accumulate=True)
    assert torch.allclose(v2, v1 + 2, atol=1e-4)
    v3 = torch.full_like(v1, 7.0)
    plan.adjoint(y, out=v3, accumulate=False)
    assert torch.equal(v3, v1)


@pytest.mark.parametrize("path", ["tma", "global"])
@pytest.mark.parametrize("case_fn", [K.c1_small, K.odd_case])
def test_pseudo_bp_matches_oracle(oracle, cuda_device, monkeypatch, case_fn, path):
    # BP_FDK_PseudoMatched through ykb_operator_apply: the TMA-staged tap-pair
    # kernel and the bounds-checked fallback against the FP64 restatement
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    if path == "global":
        monkeypatch.setenv("YKB_PSEUDO_BP_GLOBAL", "1")
    case = case_fn()
    views, plan = _plan(case)
    y = oracle.normal(plan.proj_shape, 13)
    yd = torch.from_numpy(y).cuda()
    got = plan.backproject_pseudo(yd)
    plan.check()
    ref = oracle.pseudo_bp(views, case.scan.channels, case.scan.rows,
                           K.oracle_volume(oracle, case.grid), y)
    assert K.rel_rmse(got.cpu().numpy(), ref) <= 2e-5
    # accumulate, and the task value of YK::ETask
    acc = plan.apply(L.TASK_BP_FDK_PSEUDO_MATCHED, yd, got.clone(), accumulate=True)
    assert K.rel_rmse(acc.cpu().numpy(), 2 * ref) <= 2e-5
    plan.close()


def test_operator_apply_tasks(oracle, cuda_device):
    import torch
    from fdk_cuda_impl_b200 import _lib as L
    case = K.c1_small()
    views, plan = _plan(case)
    x = torch.from_numpy(K.phantom(oracle, case)).cuda()
    assert torch.equal(plan.apply(L.TASK_FP_JOSEPH, x), plan.forward(x))
    y = plan.forward(x)
    assert torch.equal(plan.apply(L.TASK_BP_JOSEPH, y), plan.adjoint(y))
    for task in (0, 3, 5, 6, 99):
        with pytest.raises(L.YkbError) as e:
            plan.apply(task, y)
        assert e.value.code == L.ERR_UNSUPPORTED
    plan.close()


@pytest.mark.parametrize("case_fn", [K.c1_small, K.odd_case])
def test_siddon_pair_matches_oracle(oracle, cuda_device, case_fn):
    # FP_Siddon / BP_Siddon_RayDriven against the FP64 parametric Siddon, the
    # FP64 dot-product test, and accumulate
    import torch
    case = case_fn()
    views, plan = _plan(case)
    nu, nv = case.scan.channels, case.scan.rows
    vol = K.oracle_volume(oracle, case.grid)
    x = K.phantom(oracle, case)
    xd = torch.from_numpy(x).cuda()
    fp = plan.forward_siddon(xd)
    assert K.rel_rmse(fp.cpu().numpy(), oracle.siddon_fp(views, nu, nv, vol, x)) <= FP32_TOL
    y = oracle.normal(plan.proj_shape, 17)
    yd = torch.from_numpy(y).cuda()
    bp = plan.backproject_siddon(yd)
    assert K.rel_rmse(bp.cpu().numpy(), oracle.siddon_bp(views, nu, nv, vol, y)) <= FP32_TOL
    r = torch.from_numpy(oracle.uniform(case.grid.shape, 0.0, 1.0, 3)).cuda()
    lhs = float((plan.forward_siddon(r).double() * yd.double()).sum())
    rhs = float((r.double() * bp.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= ADJ_TOL
    two = plan.forward_siddon(xd, fp.clone(), accumulate=True)
    assert torch.allclose(two, 2 * fp, rtol=1e-6, atol=1e-6)
    bp2 = plan.backproject_siddon(yd, bp.clone(), accumulate=True)
    assert K.rel_rmse(bp2.cpu().numpy(), 2 * bp.cpu().numpy()) <= 1e-6
    plan.close()


@pytest.mark.parametrize("case_fn,columns", [(K.c1_small, True), (K.odd_case, False)])
def test_line_backprojector_matches_gather(oracle, cuda_device, monkeypatch, case_fn, columns):
    # axial-column scans take the line backprojector (its per-ray table is
    # four floats, so the plan's workspace grows); YKB_JOSEPH_BP=gather keeps
    # the voxel gather.  Both apply the forward projector's weights, summed
    # in different orders.  A tilted detector's columns are not axial: that
    # plan keeps the gather by itself.
    import torch
    from fdk_cuda_impl_b200.projectors import JosephPlan
    case = case_fn()
    views = case.scan.views()
    y = torch.from_numpy(oracle.normal((len(views), case.scan.rows, case.scan.channels), 12)).cuda()
    col = JosephPlan(views, case.scan.channels, case.scan.rows, case.grid)
    monkeypatch.setenv("YKB_JOSEPH_BP", "gather")
    gat = JosephPlan(views, case.scan.channels, case.scan.rows, case.grid)
    a, b = col.adjoint(y), gat.adjoint(y)
    if columns:
        assert col.workspace_bytes() > gat.workspace_bytes()
        assert K.rel_rmse(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6
    else:
        assert col.workspace_bytes() == gat.workspace_bytes()
        assert torch.equal(a, b)
    assert _adjoint_error(col, case.grid, 4) <= ADJ_TOL
    col.close()
    gat.close()


def test_line_backprojector_many_lines_per_slice(oracle, cuda_device, monkeypatch):
    # pixels an eighth of a voxel at the isocentre: a CTA slice spans about
    # 140 detector columns, so the line backprojector takes several passes of
    # 32 lines; odd volume sizes leave partial CTAs in x, y and z
    import torch
    from fdk_cuda_impl_b200.projectors import JosephPlan
    scan = CircularScan(12, 12, 300.0, 600.0, 160, 120, 0.25, 0.25)
    grid = VolumeGrid(37, 29, 21, (1.0, 1.0, 1.0))
    views = scan.views()
    y = torch.from_numpy(oracle.normal((len(views), 120, 160), 21)).cuda()
    lines = JosephPlan(views, 160, 120, grid)
    monkeypatch.setenv("YKB_JOSEPH_BP", "gather")
    gat = JosephPlan(views, 160, 120, grid)
    assert lines.workspace_bytes() > gat.workspace_bytes()
    a, b = lines.adjoint(y), gat.adjoint(y)
    assert K.rel_rmse(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6
    ref = oracle.joseph_bp(views, 160, 120, K.oracle_volume(oracle, grid), y.cpu().numpy())
    assert K.rel_rmse(a.cpu().numpy(), ref) <= FP32_TOL
    assert _adjoint_error(lines, grid, 5) <= ADJ_TOL
    lines.close()
    gat.close()
