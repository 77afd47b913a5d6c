"""Edge sizes against the FP64 oracle: a single-slice volume (nz = 1, a 2D
reconstruction), a volume thinner than one z tile, a single view, and a
detector with one row, through FDK and every projector-plan operator."""
import numpy as np
import pytest

from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter, VolumeGrid
from tests import cases as K

pytestmark = pytest.mark.gpu


def _run_all(oracle, scan, grid, fdk=True):
    import torch
    from fdk_cuda_impl_b200.projectors import FdkPlan, JosephPlan
    views = scan.views()
    nu, nv = scan.channels, scan.rows
    vol = K.oracle_volume(oracle, grid)
    x = oracle.uniform(grid.shape, 0.0, 1.0, 3)
    y = oracle.uniform((len(views), nv, nu), 0.5, 1.5, 4)
    jp = JosephPlan(views, nu, nv, grid)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    out = {
        "joseph_fp": (jp.forward(xd), oracle.joseph_fp(views, nu, nv, vol, x)),
        "joseph_bp": (jp.adjoint(yd), oracle.joseph_bp(views, nu, nv, vol, y)),
        "siddon_fp": (jp.forward_siddon(xd), oracle.siddon_fp(views, nu, nv, vol, x)),
        "siddon_bp": (jp.backproject_siddon(yd), oracle.siddon_bp(views, nu, nv, vol, y)),
        "pseudo_bp": (jp.backproject_pseudo(yd), oracle.pseudo_bp(views, nu, nv, vol, y)),
    }
    jp.check()
    jp.close()
    if fdk:
        plan = FdkPlan(views, nu, nv, scan.scan_range, grid, RampFilter())
        out["fdk"] = (plan.execute(yd), oracle.fdk(views, nu, nv, scan.scan_range, vol,
                                                   oracle.filter_struct(1), y))
        plan.check()
        plan.close()
    for name, (got, ref) in out.items():
        g = got.cpu().numpy()
        assert np.isfinite(g).all(), name
        assert K.rel_rmse(g, ref) <= 2e-5, (name, K.rel_rmse(g, ref))


@pytest.mark.parametrize("nz", [1, 5])
def test_thin_volumes(oracle, cuda_device, nz):
    scan = CircularScan(24, 24, 500.0, 1000.0, 48, 16, 1.6, 1.6)
    grid = VolumeGrid(30, 26, nz, (1.0, 1.2, 1.0))
    _run_all(oracle, scan, grid)


def test_single_view(oracle, cuda_device):
    scan = CircularScan(1, 36, 500.0, 1000.0, 40, 24, 1.6, 1.6)
    grid = VolumeGrid(20, 20, 12, (1.0, 1.0, 1.0))
    # a one-view FDK has no angular step to weight with; the projector plan
    # operators are defined for any view count
    _run_all(oracle, scan, grid, fdk=False)


def test_one_detector_row(oracle, cuda_device):
    scan = CircularScan(30, 30, 500.0, 1000.0, 40, 1, 1.6, 1.6)
    grid = VolumeGrid(24, 24, 1, (1.0, 1.0, 1.0))
    _run_all(oracle, scan, grid)
