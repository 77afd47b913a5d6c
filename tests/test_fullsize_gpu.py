"""Size-independent properties at the full workload sizes, where the FP64
oracle cannot follow: FDK linearity, the streamed host path equal to the
device-resident one, and the BF16 form against the FP32 form (<= 1e-3) on
the 512^3 x 720-view x 768^2 workload; the same at a 1024^3 volume with a
1536^2 detector (fewer views, the indexing of the large workload).

The FP32 bound is the FP32 target, 1e-5: the inputs carry a large DC part
that the ramp filter cancels, so FP32 rounding of the filter and of the view
sums shows at a few 1e-6 (2.2e-6 measured for linearity at 512^3)."""
import pytest
import torch

from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter, VolumeGrid
from fdk_cuda_impl_b200.projectors import FdkPlan

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def _rel(a, b):
    return float(((a.double() - b.double()).pow(2).mean().sqrt() / b.double().pow(2).mean().sqrt()))


def _projections(n, nv, nu, seed):
    # positive projections with structure at several scales: a bilinear
    # upsampling of uniform noise, plus 1
    g = torch.Generator(device="cuda").manual_seed(seed)
    p = torch.rand((n, nv // 8, nu // 8), device="cuda", generator=g)
    p = torch.nn.functional.interpolate(p[None], size=(nv, nu), mode="bilinear",
                                        align_corners=False)[0]
    return (1.0 + p).contiguous()


@pytest.mark.parametrize("n,views,det,vox,pix", [(512, 720, 768, 0.25, 0.4),
                                                 (1024, 96, 1536, 0.125, 0.2)])
def test_fdk_full_size_properties(cuda_device, n, views, det, vox, pix):
    scan = CircularScan(views, views, 500.0, 1000.0, det, det, pix, pix)
    grid = VolumeGrid.cube(n, vox)
    v = scan.views()
    plan = FdkPlan(v, det, det, scan.scan_range, grid, RampFilter())
    p1 = _projections(views, det, det, 1)
    p2 = _projections(views, det, det, 2)
    a = plan.execute(p1).clone()
    b = plan.execute(p2).clone()
    lin = plan.execute((2.0 * p1 - 0.5 * p2).contiguous())
    assert _rel(lin, 2.0 * a - 0.5 * b) <= FP32_TOL
    del lin, b
    # host projections in, host volume out
    host = p1.cpu().pin_memory()
    out = torch.empty(grid.shape, dtype=torch.float32).pin_memory()
    plan.execute_host(host, host_out=out)
    torch.cuda.current_stream().synchronize()
    plan.check()
    assert _rel(out, a.cpu()) <= FP32_TOL
    del host, out, a
    plan.close()
    # BF16 form on BF16-stored projections against the FP32 form on the same
    # data, both with the Shepp-Logan window
    pb = p1.to(torch.bfloat16)
    del p1, p2
    sl = RampFilter.named("shepplogan")
    ref_plan = FdkPlan(v, det, det, scan.scan_range, grid, sl)
    ref = ref_plan.execute(pb).clone()
    ref_plan.close()
    plan_b = FdkPlan(v, det, det, scan.scan_range, grid, sl, "bf16")
    got = plan_b.execute(pb)
    plan_b.check()
    assert _rel(got, ref) <= 1e-3
    plan_b.close()
