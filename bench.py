"""Benchmark: FDK backprojection GUPS on the 512^3 x 720-view workload.

Workload (the configuration the metric is quoted on): volume 512^3 of
0.25 mm voxels, 720 views over 360 deg, flat detector 768x768 of 0.4 mm,
SID/SDD 500/1000 mm, 20 seeded random ellipsoids, Poisson noise at 1e5
photons, Ram-Lak.  A step is one full FDK pass (cosine preweight + ramp
filter + weighted backprojection) over the 720 views into the volume.

value   = voxel x view updates per second of the whole job (all ranks), with
          projections already in HBM (device-timed with CUDA events).
e2e     = the same metric through the C-ABI with host buffers: each step
          copies the projections host->device (pinned) and the volume
          device->host inside the timed region.
Inputs (1.7 GB projections, 0.54 GB volume) exceed the 126 MB L2, so no
flush is needed between steps.

--impl reference times the reference's own implementation on the same
workload: its CUDA build (the reference has no CPU path), compiled for sm_100a
from its sources into oracle/_ref, through its stock FDK pipeline; the FP64
CPU oracle on a bounded sample when that build is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the headline metric: FDK GUPS is `value`; the FP+BP gradient step of the
# differentiable Joseph pair is reported beside it ("joseph")
METRIC = "FDK backprojection GUPS (voxel\u00d7view/s) & FP+BP grad step ms at stated RMSE"

# the workload the metric is quoted on, and a small case of the same kernels
# (inputs still larger than L2) used for profiler captures
# "large": the 1024^3 x 1440-view x 1536^2 FDK with BF16-stored projections
# (6.8 GB), tensor-core BF16 filter and FP32 backprojection; its phantom adds
# 200 small high-contrast spheres and it is noise-free
CONFIGS = {
    "c2": dict(N_VOX=512, N_VIEWS=720, N_DET=768, VOX_MM=0.25, PIX_MM=0.4, N_ELL=20, N_SPH=0,
               I0=1e5, PRECISION="fp32"),
    "small": dict(N_VOX=256, N_VIEWS=360, N_DET=384, VOX_MM=0.5, PIX_MM=0.8, N_ELL=20, N_SPH=0,
                  I0=1e5, PRECISION="fp32"),
    "large": dict(N_VOX=1024, N_VIEWS=1440, N_DET=1536, VOX_MM=0.125, PIX_MM=0.2, N_ELL=40,
                  N_SPH=200, I0=None, PRECISION="bf16"),
}
N_VOX = 512
N_VIEWS = 720
N_DET = 768
VOX_MM = 0.25
PIX_MM = 0.4
SID, SDD = 500.0, 1000.0
N_ELL = 20
N_SPH = 0
I0 = 1e5
PRECISION = "fp32"
UPDATES = N_VOX ** 3 * N_VIEWS
WORKLOAD = "fdk-512^3-720v-768^2"


def select_config(name: str) -> None:
    global N_VOX, N_VIEWS, N_DET, VOX_MM, PIX_MM, N_ELL, N_SPH, I0, PRECISION, UPDATES, WORKLOAD
    c = CONFIGS[name]
    N_VOX, N_VIEWS, N_DET, VOX_MM, PIX_MM = (c["N_VOX"], c["N_VIEWS"], c["N_DET"], c["VOX_MM"],
                                             c["PIX_MM"])
    N_ELL, N_SPH, I0, PRECISION = c["N_ELL"], c["N_SPH"], c["I0"], c["PRECISION"]
    UPDATES = N_VOX ** 3 * N_VIEWS
    WORKLOAD = f"fdk-{N_VOX}^3-{N_VIEWS}v-{N_DET}^2" + ("-bf16" if PRECISION == "bf16" else "")


def chunk_views() -> int:
    """Views per workspace chunk of an FDK plan: a budget of 8 GiB at 12 bytes
    per detector pixel (preweighted rows + filtered tap pairs)."""
    return max(1, min(N_VIEWS, (8 << 30) // (12 * N_DET * N_DET)))


def object_seed(rank: int) -> int:
    """Seed of rank's phantom: each rank reconstructs its own object (weak
    scaling, no data exchanged between ranks)."""
    return 1000 + rank


def max_over_ranks(x: float, world: int, device: str) -> float:
    """The slowest rank's time: all ranks take part (same collective on every
    rank), each gets the maximum."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def job_gups(world: int, updates: int, ms: float) -> float:
    """Whole-job throughput: every rank processes `updates` in the slowest
    rank's time."""
    return world * updates / (ms * 1e-3) / 1e9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-bf16", action="store_true")
    ap.add_argument("--no-joseph", action="store_true")
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    return ap.parse_args()


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        import statistics
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def cpu_baseline(n_views_sample=96, z_slab=64):
    """FP64 oracle FDK on a bounded sample of the same workload: a subset of
    views (full 768x768 projections: preweight + filter) backprojected into
    a z-slab of the volume.  Returns GUPS on the host cores."""
    import numpy as np
    from oracle import oracle as O
    views_all = O.build_circular_flat(N_VIEWS, N_VIEWS, SID, SDD, N_DET, N_DET, PIX_MM, PIX_MM)
    step = N_VIEWS // n_views_sample
    views = np.ascontiguousarray(views_all[::step][:n_views_sample])
    rng = O.regular_scan_range(N_VIEWS, N_VIEWS)
    proj = O.uniform((n_views_sample, N_DET, N_DET), 0.0, 1.0, 17)
    vol = O.volume_struct((z_slab, N_VOX, N_VOX), VOX_MM)
    filt = O.filter_struct(1)
    t0 = time.perf_counter()
    O.fdk(views, N_DET, N_DET, rng, vol, filt, proj)
    dt = time.perf_counter() - t0
    updates = n_views_sample * z_slab * N_VOX * N_VOX
    return {"value": updates / dt / 1e9, "unit": "GUPS", "cores": O.num_threads(), "kind": "port",
            "sample": f"{n_views_sample} of {N_VIEWS} views (full {N_DET}x{N_DET} preweight+ramp "
                      f"filter) backprojected into a {N_VOX}x{N_VOX}x{z_slab} slab, FP64, {dt:.1f} s"}


# Differentiable Joseph pair (the metric's "FP+BP grad step"): 256^3 of
# 0.5 mm voxels, 360 views of a 384x384 detector of 0.8 mm at 500/1000 mm
J_VOX, J_VIEWS, J_DET, J_VOX_MM, J_PIX_MM = 256, 360, 384, 0.5, 0.8


def joseph_workload():
    from fdk_cuda_impl_b200 import CircularScan, VolumeGrid
    scan = CircularScan(J_VIEWS, J_VIEWS, SID, SDD, J_DET, J_DET, J_PIX_MM, J_PIX_MM)
    return scan, VolumeGrid.cube(J_VOX, J_VOX_MM)


def joseph_step(local: int, steps: int, warmup: int, timed_fn):
    """One gradient step of 1/2 |A x - b|^2 through the autograd Joseph pair:
    y = A x (forward projector), then x.grad = A^T (y - b) (matched
    backprojector); plus the dot-product adjoint test <Ax, y> = <x, A^T y>."""
    import torch
    from fdk_cuda_impl_b200.autograd import JosephProjector
    from fdk_cuda_impl_b200.projectors import JosephPlan
    scan, grid = joseph_workload()
    plan = JosephPlan(scan.views(), J_DET, J_DET, grid, device=local)
    op = JosephProjector(plan)
    gen = torch.Generator(device=f"cuda:{local}")
    gen.manual_seed(11)
    x = torch.rand(grid.shape, device=f"cuda:{local}", generator=gen).requires_grad_(True)
    b = torch.randn(plan.proj_shape, device=f"cuda:{local}", generator=gen)

    def step():
        x.grad = None
        r = op(x) - b
        r.backward(r)  # d(1/2 |r|^2)/dr = r

    for _ in range(warmup):
        step()
    ms = timed_fn(step, steps)
    fp_ms = timed_fn(lambda: plan.forward(x.detach()), steps)
    bp_ms = timed_fn(lambda: plan.adjoint(b), steps)
    # BP_FDK_PseudoMatched, the reference's default backprojector for CGLS
    pseudo = plan.backproject_pseudo(b)
    pseudo_ms = timed_fn(lambda: plan.backproject_pseudo(b, pseudo), steps)
    plan.check()
    # the Siddon pair (FP_Siddon, BP_Siddon_RayDriven)
    sfp = plan.forward_siddon(x.detach())
    siddon_fp_ms = timed_fn(lambda: plan.forward_siddon(x.detach(), sfp), steps)
    siddon_bp_ms = timed_fn(lambda: plan.backproject_siddon(b, pseudo), steps)
    del pseudo, sfp
    with torch.no_grad():
        ax = plan.forward(x.detach())
        aty = plan.adjoint(b)
        lhs = (ax.double() * b.double()).sum().item()
        rhs = (x.detach().double() * aty.double()).sum().item()
    samples = J_VIEWS * J_DET * J_DET * J_VOX  # rays x main-axis steps
    plan.close()
    return {"workload": f"joseph-{J_VOX}^3-{J_VIEWS}v-{J_DET}^2", "grad_step_ms": ms,
            "fp_ms": fp_ms, "bp_ms": bp_ms, "adjoint_rel": abs(lhs - rhs) / abs(lhs),
            "samples_per_op": samples, "fp_gsamples": samples / (fp_ms * 1e-3) / 1e9,
            "bp_gsamples": samples / (bp_ms * 1e-3) / 1e9,
            "bp_pseudo_matched_ms": pseudo_ms,
            "bp_pseudo_matched_gups": J_VOX ** 3 * J_VIEWS / (pseudo_ms * 1e-3) / 1e9,
            "siddon_fp_ms": siddon_fp_ms, "siddon_bp_ms": siddon_bp_ms}


def make_workload(rank: int, local: int):
    """The benchmark's seeded inputs on cuda:local: ellipsoid phantom (one
    independent object per rank), Joseph forward projection, Poisson noise."""
    import torch
    from fdk_cuda_impl_b200 import CircularScan, VolumeGrid
    from fdk_cuda_impl_b200 import phantom as PH
    from fdk_cuda_impl_b200.projectors import JosephPlan
    import numpy as np
    scan = CircularScan(N_VIEWS, N_VIEWS, SID, SDD, N_DET, N_DET, PIX_MM, PIX_MM)
    grid = VolumeGrid.cube(N_VOX, VOX_MM)
    views = scan.views()
    seed = object_seed(rank)
    ell = PH.random_ellipsoids(seed, N_ELL)
    if N_SPH:
        ell = np.concatenate([ell, PH.random_spheres(seed, N_SPH)])
    phantom = PH.voxelize(grid, ell, device=f"cuda:{local}")
    dtype = torch.bfloat16 if PRECISION == "bf16" else torch.float32
    proj = torch.empty((N_VIEWS, N_DET, N_DET), dtype=dtype, device=f"cuda:{local}")
    # Joseph projection in view chunks (its plan holds a 20-byte ray record
    # per detector pixel of its views)
    step = max(1, min(N_VIEWS, (4 << 30) // (20 * N_DET * N_DET)))
    for v0 in range(0, N_VIEWS, step):
        jp = JosephPlan(views[v0:v0 + step], N_DET, N_DET, grid, device=local)
        part = jp.forward(phantom)
        if I0 is not None and dtype != torch.float32:
            PH.poisson_noise_(part, I0, seed=7 + rank + v0)
        proj[v0:v0 + step] = part
        jp.close()
        del jp, part
    del phantom
    if I0 is not None and dtype == torch.float32:
        PH.poisson_noise_(proj, I0, seed=7 + rank)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return scan, grid, views, proj


def run_reference(args):
    """The reference's own implementation of the path on the same workload.

    The reference has no CPU path (its FDK and Joseph operators are CUDA
    only), so its own implementation is its CUDA build: oracle/_ref/libykref.so,
    compiled for sm_100a from the reference sources by oracle/ref_build.py,
    driven through its stock FdkPipeline (the path its Session runs).  value =
    projections already on the device (chunked device-to-device uploads inside
    the pipeline), e2e = host projections and the volume read back, as its
    Session requires.  Without that build, the FP64 CPU oracle port is timed on
    a bounded sample instead.  Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    from oracle import ref as R
    cfg = {"workload": WORKLOAD, "volume": [N_VOX] * 3, "voxel_mm": VOX_MM, "views": N_VIEWS,
           "detector": [N_DET, N_DET], "pixel_mm": PIX_MM, "sid_sdd_mm": [SID, SDD],
           "ellipsoids": N_ELL, "noise_i0": I0, "filter": "ramlak"}
    line = {"metric": METRIC, "unit": "GUPS",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", "impl": "reference"}
    import torch
    if R.available() and torch.cuda.is_available():
        from fdk_cuda_impl_b200 import RampFilter
        scan, grid, _, proj = make_workload(0, 0)
        h_proj = proj.float().cpu().numpy()  # the reference takes FP32 projections
        del proj
        torch.cuda.empty_cache()
        ms_dev, ms_host = R.fdk_time(scan, grid, RampFilter(), h_proj, warmup=args.warmup,
                                     reps=args.steps, timeout=1800)
        value = UPDATES / (ms_dev * 1e-3) / 1e9
        cb = cpu_baseline(n_views_sample=24, z_slab=32)
        # the reference's FP_Joseph / BP_Joseph operators on the same Joseph
        # workload (each call re-uploads its texture, as its stock apply does)
        jscan, jgrid = joseph_workload()
        gen = np.random.default_rng(11)
        jx = gen.random(jgrid.shape, dtype=np.float32)
        jy = gen.standard_normal((J_VIEWS, J_DET, J_DET)).astype(np.float32)
        _, fp_ms = R.joseph_fp(jscan, jgrid, jx, warmup=args.warmup, reps=args.steps)
        _, bp_ms = R.joseph_bp(jscan, jgrid, jy, warmup=args.warmup, reps=args.steps)
        _, pseudo_ms = R.bp_pseudo(jscan, jgrid, jy, warmup=args.warmup, reps=args.steps)
        _, siddon_fp_ms = R.siddon_fp(jscan, jgrid, jx, warmup=args.warmup, reps=args.steps)
        _, siddon_bp_ms = R.siddon_bp(jscan, jgrid, jy, warmup=args.warmup, reps=args.steps)
        samples = J_VIEWS * J_DET * J_DET * J_VOX
        joseph = {"workload": f"joseph-{J_VOX}^3-{J_VIEWS}v-{J_DET}^2", "fp_ms": fp_ms,
                  "bp_ms": bp_ms, "grad_step_ms": fp_ms + bp_ms,
                  "fp_gsamples": samples / (fp_ms * 1e-3) / 1e9,
                  "bp_gsamples": samples / (bp_ms * 1e-3) / 1e9,
                  "bp_pseudo_matched_ms": pseudo_ms,
                  "bp_pseudo_matched_gups": J_VOX ** 3 * J_VIEWS / (pseudo_ms * 1e-3) / 1e9,
                  "siddon_fp_ms": siddon_fp_ms, "siddon_bp_ms": siddon_bp_ms}
        line.update({
            "value": value, "ms_per_step": ms_dev, "dtype": "f32",
            "config": dict(cfg, implementation="reference CUDA build (YKCBCT FdkPipeline, "
                           "sm_100a, -O3 -use_fast_math), oracle/_ref/libykref.so",
                           l2="inputs larger than L2"),
            "e2e": {"value": UPDATES / (ms_host * 1e-3) / 1e9, "unit": "GUPS",
                    "ms_per_step": ms_host, "h2d_bytes_per_step": int(h_proj.nbytes),
                    "d2h_bytes_per_step": int(4 * N_VOX ** 3)},
            "cpu_baseline": cb,
            "joseph": joseph,
            "gpu_launches": None,
        })
    else:
        from oracle import oracle as O  # noqa: F401  (the CPU port)
        for _ in range(args.warmup):
            cpu_baseline(n_views_sample=8, z_slab=8)
        vals = [cpu_baseline(n_views_sample=36, z_slab=32) for _ in range(args.steps)]
        value = sum(v["value"] for v in vals) / len(vals)
        cb = dict(vals[-1], value=value)
        line.update({
            "value": value, "ms_per_step": UPDATES / (value * 1e9) * 1e3, "dtype": "f64",
            "config": dict(cfg, implementation="FP64 CPU oracle port (no reference build present)",
                           sample_per_step=cb["sample"]),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        })
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    select_config(args.config)
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    from fdk_cuda_impl_b200 import CircularScan, RampFilter, VolumeGrid
    from fdk_cuda_impl_b200 import phantom as PH
    from fdk_cuda_impl_b200.projectors import FdkPlan, JosephPlan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))

    scan, grid, views, proj = make_workload(rank, local)

    plan = FdkPlan(views, N_DET, N_DET, scan.scan_range, grid, RampFilter(), PRECISION,
                   device=local)
    vol = torch.empty(grid.shape, dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / k, world, f"cuda:{local}")

    # full FDK steps, device resident
    for _ in range(args.warmup):
        plan.execute(proj, vol)
    with ClockSampler(local) as clocks:
        ms = timed(lambda: plan.execute(proj, vol), args.steps)
    clock_info = clocks.summary()
    value = job_gups(world, UPDATES, ms)

    # stage timings for the roofline (same stream, CUDA events)
    filtered = plan.filter(proj)
    for _ in range(2):
        plan.backproject(filtered, vol)
    ms_bp = timed(lambda: plan.backproject(filtered, vol), args.steps)
    ms_filter = timed(lambda: plan.filter(proj), args.steps)
    del filtered

    # end to end through the C-ABI with pinned host buffers: the projections
    # stream host -> device in batches overlapping the kernels, the volume
    # comes back to the host, all inside the timed region
    h_proj = torch.empty(proj.shape, dtype=proj.dtype, pin_memory=True)
    h_proj.copy_(proj)
    h_vol = torch.empty(grid.shape, dtype=torch.float32, pin_memory=True)
    d_in = proj
    del proj

    def e2e_step():
        plan.execute_host(h_proj, vol, host_out=h_vol)

    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    ms_e2e = timed(e2e_step, args.steps)
    e2e_value = job_gups(world, UPDATES, ms_e2e)

    # BF16 form on the same views: projections stored in BF16 (host and
    # device), Shepp-Logan window, tcgen05 split hi/lo Toeplitz filter, the
    # same backprojection.  Its error is taken against the FP32 form (itself
    # within 1e-5 of the FP64 oracle) on the same BF16-stored projections.
    bf16 = fp32_form = None
    if PRECISION == "bf16":
        # the FP32 form on the same BF16-stored projections: the error of the
        # tensor-core filter, and the speed-up it buys
        plan_s = FdkPlan(views, N_DET, N_DET, scan.scan_range, grid, RampFilter(), "fp32",
                         device=local)
        vs = torch.empty_like(vol)
        for _ in range(max(1, args.warmup - 1)):
            plan_s.execute(d_in, vs)
        ms_s = timed(lambda: plan_s.execute(d_in, vs), args.steps)
        plan.execute(d_in, vol)
        diff = (vol.double() - vs.double()).pow(2).mean().sqrt() / vs.double().pow(2).mean().sqrt()
        fp32_form = {"ms_per_step": ms_s, "gups": world * UPDATES / (ms_s * 1e-3) / 1e9,
                     "bf16_speedup": ms_s / ms, "bf16_rel_rmse_vs_fp32_form": float(diff)}
        plan_s.close()
        del vs
    elif not args.no_bf16:
        sl = RampFilter.named("shepplogan")
        plan_b = FdkPlan(views, N_DET, N_DET, scan.scan_range, grid, sl, "bf16", device=local)
        h_proj_b = torch.empty(h_proj.shape, dtype=torch.bfloat16, pin_memory=True)
        h_proj_b.copy_(h_proj)
        d_in_b = d_in.to(torch.bfloat16)
        plan_s = FdkPlan(views, N_DET, N_DET, scan.scan_range, grid, sl, "fp32", device=local)
        ref_vol = plan_s.execute(d_in_b, vol).clone()
        plan_s.close()
        vb = torch.empty_like(vol)
        for _ in range(args.warmup):
            plan_b.execute(d_in_b, vb)
        ms_b = timed(lambda: plan_b.execute(d_in_b, vb), args.steps)
        diff = (vb.double() - ref_vol.double()).pow(2).mean().sqrt() / ref_vol.double().pow(2).mean().sqrt()

        def e2e_b():
            plan_b.execute_host(h_proj_b, vb, host_out=h_vol)

        for _ in range(max(1, args.warmup - 1)):
            e2e_b()
        ms_be = timed(e2e_b, args.steps)
        bf16 = {"ms_per_step": ms_b, "gups": world * UPDATES / (ms_b * 1e-3) / 1e9,
                "speedup_vs_fp32": ms / ms_b, "rel_rmse_vs_fp32_form": float(diff),
                "e2e_ms_per_step": ms_be, "e2e_gups": world * UPDATES / (ms_be * 1e-3) / 1e9,
                "e2e_speedup_vs_fp32": ms_e2e / ms_be,
                "h2d_bytes_per_step": int(h_proj_b.numel() * 2), "filter": "shepplogan",
                "projections": "bf16"}
        plan_b.close()
        del ref_vol, vb, d_in_b, h_proj_b

    joseph = None
    if not args.no_joseph and PRECISION == "fp32":
        joseph = joseph_step(local, args.steps, args.warmup, timed)

    peaks, peak_src = measured_peaks()
    # HBM roofline of the dominant kernel (backprojection): compulsory bytes
    # per launch = filtered projections read once + volume written once.
    bp_bytes = 4.0 * N_VIEWS * N_DET * N_DET + 4.0 * N_VOX ** 3
    achieved = bp_bytes / (ms_bp * 1e-3) / 1e9
    # DRAM traffic of one launch: ncu (dram__bytes_read + write) on the
    # 256^3 x 360 x 384^2 case gave 830.8 MB against 279.4 MB compulsory
    # (tap-pair rows are 8 B per sample; L2 misses re-read some rows);
    # scaled by the compulsory bytes, which grow in proportion
    traffic = 830.8e6 * bp_bytes / (4.0 * 360 * 384 * 384 + 4.0 * 256 ** 3)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_source": peak_src,
                "traffic_source": "ncu 256^3x360x384^2 capture scaled by compulsory bytes",
                "kernel": "fdk_bp_tma_kernel<52,1,1> (TMA-staged tap pairs)", "kernel_ms": ms_bp,
                "algorithmic_bytes_per_launch": bp_bytes}
    # on-chip view of the same kernel: 16 B of bilinear taps per update
    sm_mhz = clock_info.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    onchip_peak = 148 * 128 * sm_mhz * 1e6 / 1e9  # GB/s of shared/L1 bandwidth
    onchip = {"tap_bytes_per_update": 16, "achieved_gbs": 16 * UPDATES / (ms_bp * 1e-3) / 1e9,
              "peak_gbs_nominal": onchip_peak,
              "frac": 16 * UPDATES / (ms_bp * 1e-3) / 1e9 / onchip_peak,
              "bp_gups": UPDATES / (ms_bp * 1e-3) / 1e9}

    line = {
        "metric": METRIC,
        "value": value, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if PRECISION == "fp32" else "bf16 filter, f32 backprojection",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "volume": [N_VOX] * 3, "voxel_mm": VOX_MM,
                   "views": N_VIEWS, "detector": [N_DET, N_DET], "pixel_mm": PIX_MM,
                   "sid_sdd_mm": [SID, SDD], "ellipsoids": N_ELL, "spheres": N_SPH,
                   "noise_i0": I0, "filter": "ramlak", "precision": PRECISION,
                   "projections": "bf16" if PRECISION == "bf16" else "f32",
                   "l2": f"inputs larger than L2 ({h_proj.numel() * h_proj.element_size() / 1e9:.1f} GB "
                         f"projections, {4 * N_VOX ** 3 / 1e9:.2f} GB volume)",
                   "chunk_views": chunk_views(),
                   "parallelism": f"independent objects x{world}"},
        "stages_ms": {"filter": ms_filter, "backproject": ms_bp},
        "roofline": roofline,
        "onchip": onchip,
        "e2e": {"value": e2e_value, "unit": "GUPS", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(h_proj.numel() * h_proj.element_size()),
                "d2h_bytes_per_step": int(h_vol.numel() * 4)},
        "bf16": bf16,
        "fp32_form": fp32_form,
        "joseph": joseph,
        # preweight, filter and backprojection per workspace chunk
        "gpu_launches": 3 * -(-N_VIEWS // chunk_views()) * args.steps,
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = (cpu_baseline() if N_DET <= 768 else
                                    cpu_baseline(n_views_sample=24, z_slab=32))
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"error": str(exc)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
