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
rel_rmse_vs_oracle = the FP32 volume against the FP64 oracle on a 16-slice
          slab over all views (the oracle's run is also the CPU baseline).
Inputs (1.7 GB projections, 0.54 GB volume) exceed the 126 MB L2, so no
flush is needed between steps.

Beside the headline: the BF16 form (BF16-stored projections, Shepp-Logan
window, tensor-core BF16 filter) on the same views; the 1024^3 x 1440 x 1536^2
workload with BF16-stored projections ("large", one GPU only); the
differentiable Joseph pair at 256^3 x 360 x 384^2 ("joseph").

--impl reference times the reference's own implementation on the same
workload: its CUDA build (the reference has no CPU path), compiled for sm_100a
from its sources into oracle/_ref, through its stock FDK pipeline, with inputs
from its own Joseph projector (no part of this package's library runs in that
arm); the FP64 CPU oracle on a bounded sample when that build is absent.
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
METRIC = "FDK backprojection GUPS (voxel×view/s) & FP+BP grad step ms at stated RMSE"

# z slab [z0, z0 + nz) of each workload that the FP64 oracle reconstructs:
# off-centre for the 512^3 workload (its rays cross about 70 detector rows),
# the centre for the 1024^3 one (a few rows: the oracle's direct-convolution
# filter is the cost)
PARITY_SLABS = {"c2": (384, 16), "small": (192, 16), "det768": (192, 16), "large": (510, 4)}
FILTERS = {"f32": "ramlak", "bf16": "shepplogan"}
# timed steps of the 1024^3 workload (1.3 s each) within the default run
LARGE_STEPS, LARGE_WARMUP = 3, 3


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


def bench_config(w, world: int) -> dict:
    """The workload description both arms report (one dict, same keys and
    values, so the two lines are comparable)."""
    return dict(w.describe(), filter=FILTERS[w.projections], host_memory="pinned",
                l2=f"inputs larger than L2 ({w.n_views * w.n_det ** 2 * (2 if w.projections == 'bf16' else 4) / 1e9:.1f} GB "
                   f"projections, {4 * w.n_vox ** 3 / 1e9:.2f} GB volume)",
                parallelism=f"independent objects x{world}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-bf16", action="store_true")
    ap.add_argument("--no-joseph", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--config", default="c2", choices=["c2", "small", "det768", "large"])
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


def rel_rmse(a, ref) -> float:
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.sqrt(np.mean((a - ref) ** 2)) / max(np.sqrt(np.mean(ref ** 2)), 1e-300))


# ----------------------------------------------------------- CPU baseline ---
def cpu_baseline_leg(w, views, scan_range, forms):
    """The FP64 CPU oracle (a restatement of the reference FDK) on a bounded
    sample of workload w, timed on the host cores: all views, preweighted and
    filtered on the detector rows that the parity slab reads, backprojected
    into that slab.  The same oracle volumes check the GPU results.

    forms: {name: (host projections [views][rows][cols] tensor or array,
    filter name, GPU slab or None)}.  Returns (cpu_baseline of the first
    form, {name: rel RMSE of its GPU slab against the oracle})."""
    import numpy as np
    from oracle import oracle as O
    from fdk_cuda_impl_b200.geometry import RampFilter
    from fdk_cuda_impl_b200.workloads import slab
    z0, nz = PARITY_SLABS[w.name]
    g = slab(w, z0, nz)
    vol = O.volume_struct(g.shape, g.voxel_mm, g.center_mm)
    r0, nr = O.fdk_row_band(views, w.n_det, w.n_det, scan_range, vol)
    baseline, errors = None, {}
    for name, (host_proj, filt, gpu_slab) in forms.items():
        rows = host_proj[:, r0:r0 + nr, :]
        rows = np.ascontiguousarray(rows.float().numpy() if hasattr(rows, "float") else rows,
                                    dtype=np.float32)
        f = RampFilter.named(filt)
        of = O.filter_struct(f.type, f.cutoff, f.gain, f.butterworth_order, f.kaiser_beta,
                             f.tukey_alpha)
        t0 = time.perf_counter()
        ref = O.fdk_rows(views, w.n_det, w.n_det, scan_range, vol, of, rows, r0)
        dt = time.perf_counter() - t0
        if baseline is None:
            updates = w.n_views * nz * w.n_vox * w.n_vox
            baseline = {"value": updates / dt / 1e9, "unit": "GUPS", "cores": O.num_threads(),
                        "kind": "port",
                        "sample": f"all {w.n_views} views (preweight + {filt} filter of the "
                                  f"{nr} detector rows the slab reads) backprojected into slices "
                                  f"{z0}..{z0 + nz - 1} ({w.n_vox}x{w.n_vox}x{nz}), FP64, "
                                  f"{dt:.1f} s"}
        if gpu_slab is not None:
            errors[name] = rel_rmse(gpu_slab, ref)
    return baseline, errors


# ------------------------------------------------------------ Joseph pair ---
# Differentiable Joseph pair (the metric's "FP+BP grad step"): 256^3 of
# 0.5 mm voxels, 360 views of a 384x384 detector of 0.8 mm at 500/1000 mm
J_VOX, J_VIEWS, J_DET, J_VOX_MM, J_PIX_MM = 256, 360, 384, 0.5, 0.8


def joseph_workload():
    from fdk_cuda_impl_b200.geometry import CircularScan, VolumeGrid
    scan = CircularScan(J_VIEWS, J_VIEWS, 500.0, 1000.0, J_DET, J_DET, J_PIX_MM, J_PIX_MM)
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


# -------------------------------------------------------- reference arm ---
def run_reference(args):
    """The reference's own implementation of the path on the same workload.

    The reference has no CPU path (its FDK and Joseph operators are CUDA
    only), so its own implementation is its CUDA build: oracle/_ref/libykref.so,
    compiled for sm_100a from the reference sources by oracle/ref_build.py,
    driven through its stock FdkPipeline (the path its Session runs).  Its
    inputs come from the same seeded phantom projected by its own FP_Joseph;
    views for the oracle come from the oracle's builder (bit-identical to the
    reference builders).  Nothing of this package's library runs here.
    value = projections already on the device (chunked device-to-device
    uploads inside the pipeline), e2e = pinned host projections in and the
    volume read back to pinned host memory, as its Session's host path does.
    Without that build, the FP64 CPU oracle port is timed on a bounded sample
    instead.  Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import numpy as np
    import torch
    from oracle import oracle as O
    from oracle import ref as R
    from fdk_cuda_impl_b200.geometry import RampFilter
    from fdk_cuda_impl_b200.workloads import WORKLOADS, make_projections
    w = WORKLOADS[args.config]
    line = {"metric": METRIC, "unit": "GUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "impl": "reference",
            "config": bench_config(w, world)}
    if not (R.available() and torch.cuda.is_available()):
        scan = w.scan()
        views = O.build_circular_flat(w.n_views, w.n_views, scan.sid_mm, scan.sdd_mm, w.n_det,
                                      w.n_det, w.pix_mm, w.pix_mm)
        host = O.uniform((w.n_views, w.n_det, w.n_det), 0.0, 1.0, 17)
        cb, _ = cpu_baseline_leg(w, views, O.regular_scan_range(w.n_views, w.n_views),
                                 {"f32": (host, FILTERS[w.projections], None)})
        line.update({"value": cb["value"], "ms_per_step": w.updates / (cb["value"] * 1e9) * 1e3,
                     "dtype": "f64", "cpu_baseline": cb,
                     "implementation": "FP64 CPU oracle port (no reference build present)",
                     "e2e": {"value": cb["value"], "unit": "GUPS", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        print(json.dumps(line), flush=True)
        return

    def reference_fdk(w, seed, warmup, steps):
        scan, grid = w.scan(), w.grid()
        views = O.build_circular_flat(w.n_views, w.n_views, scan.sid_mm, scan.sdd_mm, w.n_det,
                                      w.n_det, w.pix_mm, w.pix_mm)
        scan_range = O.regular_scan_range(w.n_views, w.n_views)

        def ref_forward(_views, phantom):
            out, _ = R.joseph_fp(scan, grid, phantom.cpu().numpy())
            return torch.from_numpy(out).cuda()

        _, proj = make_projections(w, seed, 0, forward=ref_forward, views=views,
                                   chunk_views=w.n_views)
        # the reference takes FP32 projections (BF16-stored ones widen exactly)
        h_proj = proj.float().cpu().numpy()
        del proj
        torch.cuda.empty_cache()
        filt = RampFilter.named(FILTERS[w.projections])
        ms_dev, ms_host, vol = R.fdk_time(scan, grid, filt, h_proj, warmup=warmup, reps=steps,
                                          timeout=1800)
        z0, nz = PARITY_SLABS[w.name]
        cb, err = cpu_baseline_leg(w, views, scan_range,
                                   {"f32": (h_proj, FILTERS[w.projections], vol[z0:z0 + nz])})
        return ms_dev, ms_host, h_proj.nbytes, cb, err["f32"]

    ms_dev, ms_host, h2d, cb, err = reference_fdk(w, object_seed(0), args.warmup, args.steps)
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
        "value": w.updates / (ms_dev * 1e-3) / 1e9, "ms_per_step": ms_dev, "dtype": "f32",
        "implementation": "reference CUDA build (YKCBCT FdkPipeline, sm_100a, -O3 "
                          "-use_fast_math), oracle/_ref/libykref.so; inputs from its FP_Joseph",
        "rel_rmse_vs_oracle": err,
        "e2e": {"value": w.updates / (ms_host * 1e-3) / 1e9, "unit": "GUPS",
                "ms_per_step": ms_host, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(4 * w.n_vox ** 3)},
        "cpu_baseline": cb,
        "joseph": joseph,
        "gpu_launches": None,
    })
    if args.config == "c2" and not args.no_large:
        # the 1024^3 workload, FP32 projections (the reference stores no BF16)
        wl = WORKLOADS["large"]
        try:
            l_dev, l_host, l_h2d, _, l_err = reference_fdk(wl, object_seed(0), LARGE_WARMUP,
                                                           LARGE_STEPS)
            line["large"] = {"config": bench_config(wl, world), "steps": LARGE_STEPS,
                             "warmup": LARGE_WARMUP,
                             "gups": wl.updates / (l_dev * 1e-3) / 1e9, "ms_per_step": l_dev,
                             "e2e_gups": wl.updates / (l_host * 1e-3) / 1e9,
                             "e2e_ms_per_step": l_host, "h2d_bytes_per_step": int(l_h2d),
                             "rel_rmse_vs_oracle": l_err, "projections_given": "f32"}
        except Exception as exc:  # reported, never required
            line["large"] = {"error": str(exc)}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- our arm ---
def stage_times(plan, step, steps):
    """Per launch group device times (ms) of the filter and the
    backprojection inside `steps` calls of `step` (ykb_fdk_stage_timing)."""
    plan.stage_timing(True)
    for _ in range(steps):
        step()
    t = plan.stage_times()
    plan.stage_timing(False)
    return {"filter_ms": t["filter_ms"] / max(t["filter_groups"], 1),
            "backproject_ms": t["backproject_ms"] / max(t["backproject_groups"], 1),
            "groups_per_step": t["backproject_groups"] / steps}


def fdk_form(plan, d_proj, h_proj, vol, h_vol, steps, warmup, timed, slab):
    """Device-resident and end-to-end timings of one FDK plan; returns
    (ms, e2e ms, host copy of the parity slab of the device-resident volume)."""
    for _ in range(warmup):
        plan.execute(d_proj, vol)
    ms = timed(lambda: plan.execute(d_proj, vol), steps)
    plan.check()
    z0, nz = slab
    gpu_slab = vol[z0:z0 + nz].cpu().numpy()

    def e2e():
        plan.execute_host(h_proj, vol, host_out=h_vol)

    for _ in range(max(1, warmup - 1)):
        e2e()
    ms_e2e = timed(e2e, steps)
    plan.check()
    return ms, ms_e2e, gpu_slab


def large_block(world, rank, local, timed, cpu_leg: bool):
    """The 1024^3 x 1440 x 1536^2 workload, BF16-stored projections: the BF16
    form (tensor-core BF16 filter, FP32 backprojection) device-resident and
    end to end, the FP32 form on the same data, both against the oracle."""
    import torch
    from fdk_cuda_impl_b200.geometry import RampFilter
    from fdk_cuda_impl_b200.projectors import FdkPlan
    from fdk_cuda_impl_b200.workloads import WORKLOADS, make_projections
    w = WORKLOADS["large"]
    scan, grid = w.scan(), w.grid()
    views, proj = make_projections(w, object_seed(rank), local)
    sl = RampFilter.named(FILTERS[w.projections])
    plan = FdkPlan(views, w.n_det, w.n_det, scan.scan_range, grid, sl, "bf16", device=local)
    vol = torch.empty(grid.shape, dtype=torch.float32, device=f"cuda:{local}")
    h_proj = torch.empty(proj.shape, dtype=proj.dtype, pin_memory=True)
    h_proj.copy_(proj)
    h_vol = torch.empty(grid.shape, dtype=torch.float32, pin_memory=True)
    slab = PARITY_SLABS[w.name]
    ms, ms_e2e, slab_b = fdk_form(plan, proj, h_proj, vol, h_vol, LARGE_STEPS, LARGE_WARMUP,
                                  timed, slab)
    stages = stage_times(plan, lambda: plan.execute(proj, vol), LARGE_STEPS)
    plan.check()
    plan.close()
    torch.cuda.empty_cache()
    plan_s = FdkPlan(views, w.n_det, w.n_det, scan.scan_range, grid, sl, "fp32", device=local)
    plan_s.execute(proj, vol)
    ms_s = timed(lambda: plan_s.execute(proj, vol), LARGE_STEPS)
    plan_s.check()
    slab_s = vol[slab[0]:slab[0] + slab[1]].cpu().numpy()
    plan_s.close()
    del proj, vol
    torch.cuda.empty_cache()
    out = {"config": bench_config(w, world), "steps": LARGE_STEPS, "warmup": LARGE_WARMUP,
           "ms_per_step": ms, "gups": job_gups(world, w.updates, ms),
           "e2e_ms_per_step": ms_e2e, "e2e_gups": job_gups(world, w.updates, ms_e2e),
           "h2d_bytes_per_step": int(h_proj.numel() * 2), "d2h_bytes_per_step": int(h_vol.numel() * 4),
           "stages_ms_per_launch": stages,
           "backproject_gups": w.updates / (stages["backproject_ms"] * stages["groups_per_step"]
                                            * 1e-3) / 1e9,
           "fp32_form": {"ms_per_step": ms_s, "gups": job_gups(world, w.updates, ms_s),
                         "bf16_speedup": ms_s / ms}}
    if cpu_leg:
        cb, err = cpu_baseline_leg(w, views, scan.scan_range,
                                   {"bf16": (h_proj, FILTERS[w.projections], slab_b),
                                    "fp32": (h_proj, FILTERS[w.projections], slab_s)})
        out["rel_rmse_vs_oracle"] = err["bf16"]
        out["fp32_form"]["rel_rmse_vs_oracle"] = err["fp32"]
        out["oracle_slab"] = list(slab)
        out["cpu_baseline"] = cb
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    from fdk_cuda_impl_b200 import _lib as L
    from fdk_cuda_impl_b200.geometry import RampFilter
    from fdk_cuda_impl_b200.projectors import FdkPlan
    from fdk_cuda_impl_b200.workloads import WORKLOADS, make_projections

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
    w = WORKLOADS[args.config]
    scan, grid = w.scan(), w.grid()
    views, proj = make_projections(w, object_seed(rank), local)
    precision = "bf16" if w.projections == "bf16" else "fp32"
    filt = RampFilter.named(FILTERS[w.projections])
    plan = FdkPlan(views, w.n_det, w.n_det, scan.scan_range, grid, filt, precision, device=local)
    vol = torch.empty(grid.shape, dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    slab = PARITY_SLABS[w.name]

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
    plan.check()
    clock_info = clocks.summary()
    value = job_gups(world, w.updates, ms)
    gpu_slab = vol[slab[0]:slab[0] + slab[1]].cpu().numpy()

    # stage timings for the roofline: CUDA events around the filter and the
    # backprojection launch groups inside full steps, on the launching stream
    stages = stage_times(plan, lambda: plan.execute(proj, vol), args.steps)
    ms_bp, ms_filter = stages["backproject_ms"], stages["filter_ms"]
    plan.check()

    # end to end through the C-ABI with pinned host buffers: the projections
    # stream host -> device in batches overlapping the kernels, the volume
    # comes back to the host, all inside the timed region
    h_proj = torch.empty(proj.shape, dtype=proj.dtype, pin_memory=True)
    h_proj.copy_(proj)
    h_vol = torch.empty(grid.shape, dtype=torch.float32, pin_memory=True)

    def e2e_step():
        plan.execute_host(h_proj, vol, host_out=h_vol)

    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    ms_e2e = timed(e2e_step, args.steps)
    plan.check()
    e2e_value = job_gups(world, w.updates, ms_e2e)
    plan.close()

    # BF16 form on the same views: projections stored in BF16 (host and
    # device), Shepp-Logan window, tcgen05 split hi/lo Toeplitz filter, the
    # same backprojection; against the FP64 oracle on the same BF16-stored
    # projections (cpu leg) and against the FP32 form on them
    bf16 = None
    h_proj_b = None
    if precision == "fp32" and not args.no_bf16:
        sl = RampFilter.named("shepplogan")
        d_in_b = proj.to(torch.bfloat16)
        plan_s = FdkPlan(views, w.n_det, w.n_det, scan.scan_range, grid, sl, "fp32", device=local)
        ref_vol = plan_s.execute(d_in_b, vol).clone()
        plan_s.check()
        plan_s.close()
        plan_b = FdkPlan(views, w.n_det, w.n_det, scan.scan_range, grid, sl, "bf16", device=local)
        h_proj_b = torch.empty(h_proj.shape, dtype=torch.bfloat16, pin_memory=True)
        h_proj_b.copy_(d_in_b)
        vb = torch.empty_like(vol)
        ms_b, ms_be, gpu_slab_b = fdk_form(plan_b, d_in_b, h_proj_b, vb, h_vol, args.steps,
                                           args.warmup, timed, slab)
        diff = (vb.double() - ref_vol.double()).pow(2).mean().sqrt() / ref_vol.double().pow(2).mean().sqrt()
        bf16 = {"ms_per_step": ms_b, "gups": job_gups(world, w.updates, ms_b),
                "speedup_vs_fp32": ms / ms_b, "rel_rmse_vs_fp32_form": float(diff),
                "e2e_ms_per_step": ms_be, "e2e_gups": job_gups(world, w.updates, ms_be),
                "e2e_speedup_vs_fp32": ms_e2e / ms_be,
                "h2d_bytes_per_step": int(h_proj_b.numel() * 2), "filter": "shepplogan",
                "projections": "bf16"}
        plan_b.close()
        del ref_vol, vb, d_in_b
    del proj
    torch.cuda.empty_cache()

    joseph = None
    if not args.no_joseph and args.config == "c2":
        joseph = joseph_step(local, args.steps, args.warmup, timed)

    peaks, peak_src = measured_peaks()
    # HBM roofline of the dominant kernel (backprojection): compulsory bytes
    # per step = filtered projections read once + volume written once, spread
    # over the step's launches (one at the 512^3 x 720 workload)
    bp_step_ms = ms_bp * stages["groups_per_step"]
    bp_bytes = 4.0 * w.n_views * w.n_det ** 2 + 4.0 * w.n_vox ** 3
    achieved = bp_bytes / (bp_step_ms * 1e-3) / 1e9
    # DRAM traffic of one launch: ncu (dram__bytes_read + write) on the
    # 256^3 x 360 x 384^2 case gave 703.4 + 64.8 MB against 279.4 MB
    # compulsory (tap-pair rows are 8 B per sample; L2 misses re-read some
    # rows); scaled by the compulsory bytes of one launch, which grow in
    # proportion
    traffic = 768.2e6 * (bp_bytes / stages["groups_per_step"]) / (
        4.0 * 360 * 384 * 384 + 4.0 * 256 ** 3)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_source": peak_src,
                "traffic_source": "ncu 256^3x360x384^2 capture scaled by compulsory bytes",
                "kernel": "fdk_bp_tma_kernel (TMA-staged tap pairs)", "kernel_ms": ms_bp,
                "kernel_ms_source": "CUDA events around its launch inside the FDK steps",
                "algorithmic_bytes_per_launch": bp_bytes / stages["groups_per_step"]}
    # the bound that binds: 16 B of bilinear taps per update, loaded from
    # shared memory as two 8-byte tap pairs, against the measured 8-byte
    # shared-load bandwidth of this GPU
    import ctypes as C
    smem = C.c_double(0.0)
    smem_status = L.load().ykb_measure_shared_load_gbs(local, 8, C.byref(smem))
    tap_gbs = 16 * w.updates / (bp_step_ms * 1e-3) / 1e9
    onchip = {"tap_bytes_per_update": 16, "achieved_gbs": tap_gbs,
              "bp_gups": w.updates / (bp_step_ms * 1e-3) / 1e9}
    if smem_status == L.OK:
        onchip.update({"peak_gbs": smem.value, "frac": tap_gbs / smem.value,
                       "peak_source": "measured: ykb_measure_shared_load_gbs, 8-byte "
                                      "conflict-free shared loads, 4 CTAs per SM"})
    else:
        onchip["peak_error"] = L.load().ykb_last_error().decode()

    line = {
        "metric": METRIC,
        "value": value, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if precision == "fp32" else "bf16 filter, f32 backprojection",
        "data": "synthetic",
        "config": bench_config(w, world),
        "stages_ms": {"filter": ms_filter, "backproject": ms_bp,
                      "launches_per_step": stages["groups_per_step"],
                      "how": "CUDA events around each launch group inside full steps"},
        "roofline": roofline,
        "onchip": onchip,
        "e2e": {"value": e2e_value, "unit": "GUPS", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(h_proj.numel() * h_proj.element_size()),
                "d2h_bytes_per_step": int(h_vol.numel() * 4)},
        "bf16": bf16,
        "joseph": joseph,
        # preweight, filter and backprojection per workspace chunk
        "gpu_launches": 3 * -(-w.n_views // plan_chunk_views(w)) * args.steps,
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            forms = {"f32": (h_proj, FILTERS[w.projections], gpu_slab)}
            if h_proj_b is not None:
                forms["bf16"] = (h_proj_b, "shepplogan", gpu_slab_b)
            cb, err = cpu_baseline_leg(w, views, scan.scan_range, forms)
            line["cpu_baseline"] = cb
            line["rel_rmse_vs_oracle"] = err["f32"]
            line["oracle_slab"] = list(slab)
            if bf16 is not None:
                bf16["rel_rmse_vs_oracle"] = err["bf16"]
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"error": str(exc)}
    del h_proj, h_proj_b, h_vol
    if world == 1 and args.config == "c2" and not args.no_large:
        try:
            line["large"] = large_block(world, rank, local, timed,
                                        cpu_leg=rank == 0 and not args.no_cpu_baseline)
        except Exception as exc:
            line["large"] = {"error": str(exc)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def plan_chunk_views(w) -> int:
    """Views per workspace chunk of an FDK plan: a budget of 8 GiB at 12 bytes
    per detector pixel (preweighted rows + filtered tap pairs)."""
    return max(1, min(w.n_views, (8 << 30) // (12 * w.n_det * w.n_det)))


if __name__ == "__main__":
    main()
