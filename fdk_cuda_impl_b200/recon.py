"""Gradient-based reconstruction through the differentiable Joseph pair.

The consumers of the FP/BP operators that the reference drives from its
iterative solvers (src/Reconstruction/Iterative/Flat/YkCglsBackends.hpp:22-196):

* ``cgls``: CGLS with the Joseph pair and FP64 dot products, the algorithm of
  the reference's ``CglsAstraBackend::run`` (:70-150), on the library's
  vector kernels (``IterVectors``).  The reference reduces its dots in FP32
  and synchronises the host on each one; here the loop never waits on the
  host.
* ``unrolled_tv``: TV-regularised reconstruction by differentiating through
  unrolled iterations.  K gradient iterations
      x_{k+1} = x_k - alpha_k (A^T (A x_k - b) / m + lam grad TV(x_k))
  start from x_0.  Adam adjusts x_0 and the step sizes alpha_k (kept positive
  through their logarithms) to minimise the objective of the last iterate,
      L(x_K) = 1/2 mean((A x_K - b)^2) + lam mean(TV(x_K)),
  with both means reduced in FP64.  The objective is normalised by the ray and
  voxel counts so that lam is independent of the problem size.  Each unrolled
  iteration runs under ``torch.utils.checkpoint``: only the K iterates are
  kept, and the backward pass recomputes each iteration's projections.

TV is isotropic: sqrt(dx^2 + dy^2 + dz^2 + eps^2) with forward differences
and a zero difference across the far faces.  Its gradient is written out
explicitly, so each unrolled step is first-order in torch ops.
"""
from __future__ import annotations

import ctypes as C
import math

import torch
from torch.utils.checkpoint import checkpoint

from . import _lib as L
from .autograd import JosephProjector
from .projectors import JosephPlan

TV_EPS = 1e-4


def _diffs(x: torch.Tensor):
    # forward differences along z, y, x of a [z][y][x] volume, zero at the far face
    dz = torch.zeros_like(x)
    dy = torch.zeros_like(x)
    dx = torch.zeros_like(x)
    dz[:-1] = x[1:] - x[:-1]
    dy[:, :-1] = x[:, 1:] - x[:, :-1]
    dx[:, :, :-1] = x[:, :, 1:] - x[:, :, :-1]
    return dz, dy, dx


def tv(x: torch.Tensor, eps: float = TV_EPS) -> torch.Tensor:
    """mean over voxels of sqrt(|grad x|^2 + eps^2), reduced in FP64."""
    dz, dy, dx = _diffs(x)
    return torch.sqrt(dz * dz + dy * dy + dx * dx + eps * eps).double().mean()


def tv_grad(x: torch.Tensor, eps: float = TV_EPS) -> torch.Tensor:
    """Gradient of sum sqrt(|grad x|^2 + eps^2): the negative divergence of
    the normalised gradient field (the adjoint of the forward differences)."""
    dz, dy, dx = _diffs(x)
    n = torch.sqrt(dz * dz + dy * dy + dx * dx + eps * eps)
    pz, py, px = dz / n, dy / n, dx / n
    g = torch.zeros_like(x)
    # adjoint of the forward difference: (D^T p)[i] = p[i-1] - p[i]
    g -= pz
    g[1:] += pz[:-1]
    g -= py
    g[:, 1:] += py[:, :-1]
    g -= px
    g[:, :, 1:] += px[:, :, :-1]
    return g


def data_loss(ax: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    r = (ax - b).double()
    return 0.5 * (r * r).mean()


def objective(op: JosephProjector, x: torch.Tensor, b: torch.Tensor, lam: float) -> torch.Tensor:
    return data_loss(op(x), b) + lam * tv(x)


def power_norm(plan: JosephPlan, iters: int = 8, seed: int = 0) -> float:
    """||A||^2 by power iteration on A^T A."""
    g = torch.Generator(device=f"cuda:{plan.device}")
    g.manual_seed(seed)
    x = torch.rand(plan.grid.shape, device=f"cuda:{plan.device}", generator=g)
    lam = 0.0
    for _ in range(iters):
        y = plan.adjoint(plan.forward(x))
        lam = float(torch.linalg.vector_norm(y.double()) / torch.linalg.vector_norm(x.double()))
        x = y / torch.linalg.vector_norm(y)
    return lam


class IterVectors:
    """The library's vector kernels for iterative solvers (ykb_iter_*): FP64
    dot products written on the device and CGLS updates whose step sizes
    are read there, so a solver loop never waits on the host."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        self.device = device
        h = C.c_void_p()
        L.check(self.lib.ykb_iter_create(device, C.byref(h)))
        self._h = h

    def dot(self, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """out (a float64 device scalar) = sum a * b in FP64."""
        assert a.is_contiguous() and b.is_contiguous() and a.numel() == b.numel()
        assert out.dtype == torch.float64 and out.numel() == 1
        L.check(self.lib.ykb_dot_f64(self._h, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                     a.numel(), C.c_void_p(out.data_ptr()), _stream(self.device)))
        return out

    def update_xr(self, gamma, ww, x, p, r, w) -> None:
        """x += (gamma / ww) p,  r -= (gamma / ww) w."""
        L.check(self.lib.ykb_cgls_update_xr(self._h, C.c_void_p(gamma.data_ptr()),
                                            C.c_void_p(ww.data_ptr()), C.c_void_p(x.data_ptr()),
                                            C.c_void_p(p.data_ptr()), x.numel(),
                                            C.c_void_p(r.data_ptr()), C.c_void_p(w.data_ptr()),
                                            r.numel(), _stream(self.device)))

    def update_p(self, gamma_new, gamma_old, p, z) -> None:
        """p = z + (gamma_new / gamma_old) p."""
        L.check(self.lib.ykb_cgls_update_p(self._h, C.c_void_p(gamma_new.data_ptr()),
                                           C.c_void_p(gamma_old.data_ptr()),
                                           C.c_void_p(p.data_ptr()), C.c_void_p(z.data_ptr()),
                                           p.numel(), _stream(self.device)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.ykb_iter_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream(device: int):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def cgls(plan: JosephPlan, b: torch.Tensor, n_iter: int, x0: torch.Tensor | None = None):
    """CGLS for min ||A x - b||^2 (the algorithm of the reference's
    CglsAstraBackend::run) with FP64 dot products on the device.  The loop
    enqueues work only: step sizes stay on the device (ykb_cgls_update_*),
    and the residual norms are read once at the end.  Returns (x, residual
    norms per iteration)."""
    vec = IterVectors(plan.device)
    dev = b.device
    x = torch.zeros(plan.grid.shape, device=dev) if x0 is None else x0.clone()
    r = b - plan.forward(x)
    p = plan.adjoint(r)
    w = torch.empty_like(r)
    z = torch.empty_like(p)
    # scalars: gamma for each iteration, |w|^2, |r|^2 per iteration
    gamma = torch.zeros(n_iter + 1, dtype=torch.float64, device=dev)
    ww = torch.zeros(1, dtype=torch.float64, device=dev)
    rr = torch.zeros(n_iter + 1, dtype=torch.float64, device=dev)
    vec.dot(p, p, gamma[0:1])
    vec.dot(r, r, rr[0:1])
    for k in range(n_iter):
        plan.forward(p, w)
        vec.dot(w, w, ww)
        vec.update_xr(gamma[k:k + 1], ww, x, p, r, w)
        plan.adjoint(r, z)
        vec.dot(z, z, gamma[k + 1:k + 2])
        vec.update_p(gamma[k + 1:k + 2], gamma[k:k + 1], p, z)
        vec.dot(r, r, rr[k + 1:k + 2])
    norms = [float(v) for v in torch.sqrt(rr).cpu()]
    vec.close()
    return x, norms


class UnrolledTV(torch.nn.Module):
    """K unrolled gradient iterations on the TV-regularised objective, with a
    learnable start x_0 and learnable step sizes alpha_k = exp(log_alpha_k).

    momentum=True runs the iterations with the FISTA extrapolation
        y_k = x_k + (t_{k-1} - 1) / t_k (x_k - x_{k-1}),  x_{k+1} = y_k - alpha_k g(y_k)
    (Beck and Teboulle, 2009), which reaches the higher frequencies of the
    data term in fewer iterations than plain gradient steps."""

    def __init__(self, plan: JosephPlan, b: torch.Tensor, n_unrolled: int = 10,
                 lam: float = 1e-3, alpha0: float | None = None, use_checkpoint: bool = True,
                 x_init: torch.Tensor | None = None, momentum: bool = False):
        super().__init__()
        self.plan, self.op = plan, JosephProjector(plan)
        self.register_buffer("b", b)
        self.lam, self.use_checkpoint, self.momentum = lam, use_checkpoint, momentum
        self.m = b.numel()
        if alpha0 is None:
            # 1/L of the normalised data term, L = ||A||^2 / m
            alpha0 = self.m / power_norm(plan)
        x0 = torch.zeros(plan.grid.shape, device=b.device) if x_init is None else x_init.clone()
        self.x0 = torch.nn.Parameter(x0)
        self.log_alpha = torch.nn.Parameter(
            torch.full((n_unrolled,), math.log(alpha0), device=b.device))
        t = [1.0]
        for _ in range(n_unrolled):
            t.append((1.0 + math.sqrt(1.0 + 4.0 * t[-1] ** 2)) / 2.0)
        self.beta = [(t[k] - 1.0) / t[k + 1] for k in range(n_unrolled)]

    def grad(self, x: torch.Tensor) -> torch.Tensor:
        r = self.op(x) - self.b
        return self.op.adjoint(r) / self.m + self.lam * tv_grad(x) / x.numel()

    def _step(self, x: torch.Tensor, log_alpha: torch.Tensor) -> torch.Tensor:
        return x - torch.exp(log_alpha) * self.grad(x)

    def _step_momentum(self, x: torch.Tensor, x_prev: torch.Tensor, log_alpha: torch.Tensor,
                       beta: float):
        y = x + beta * (x - x_prev)
        return y - torch.exp(log_alpha) * self.grad(y), x

    def forward(self) -> torch.Tensor:
        x = x_prev = self.x0
        for k in range(self.log_alpha.numel()):
            if self.momentum:
                args = (x, x_prev, self.log_alpha[k], self.beta[k])
                if self.use_checkpoint:
                    x, x_prev = checkpoint(self._step_momentum, *args, use_reentrant=False)
                else:
                    x, x_prev = self._step_momentum(*args)
            elif self.use_checkpoint:
                x = checkpoint(self._step, x, self.log_alpha[k], use_reentrant=False)
            else:
                x = self._step(x, self.log_alpha[k])
        return x

    def loss(self, x: torch.Tensor) -> torch.Tensor:
        return objective(self.op, x, self.b, self.lam)


def unrolled_tv(plan: JosephPlan, b: torch.Tensor, adam_steps: int = 50, n_unrolled: int = 10,
                lam: float = 1e-3, lr: float | None = None, lr_rel: float = 0.01,
                use_checkpoint: bool = True, x_init: torch.Tensor | None = None,
                momentum: bool = True, callback=None):
    """Runs the Adam outer loop; returns (x_K, model, losses).

    Adam moves every voxel by about lr per step whatever its gradient's
    size, so lr is a voxel value: by default lr_rel times the RMS voxel value
    of the unrolled iterate before optimisation."""
    model = UnrolledTV(plan, b, n_unrolled, lam, use_checkpoint=use_checkpoint, x_init=x_init,
                       momentum=momentum)
    if lr is None:
        with torch.no_grad():
            lr = lr_rel * float(torch.sqrt((model().double() ** 2).mean()))
    opt = torch.optim.Adam([{"params": [model.x0], "lr": lr},
                            {"params": [model.log_alpha], "lr": 0.05}])
    losses = []
    for it in range(adam_steps):
        opt.zero_grad(set_to_none=True)
        xk = model()
        loss = model.loss(xk)
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
        if callback is not None:
            callback(it, losses[-1])
    with torch.no_grad():
        xk = model()
    return xk.detach(), model, losses


def make_problem(n: int = 256, n_views: int = 90, det: int = 384, vox: float = 0.5,
                 pix: float = 0.8, i0: float = 5e4, seed: int = 4, device: int = 0):
    """Noisy sparse-view problem: a random-ellipsoid phantom on an n^3 grid,
    n_views views over a full turn on a det^2 detector, Poisson noise at I0
    photons.  Attenuation is scaled so that the longest line integral is 3
    (5 % of the photons transmitted), which keeps the noise model in its
    linear range instead of saturating at ln(I0).
    Returns (scan, grid, plan, truth, b)."""
    from . import phantom as PH
    from .geometry import CircularScan, VolumeGrid
    scan = CircularScan(n_views, n_views, 500.0, 1000.0, det, det, pix, pix)
    grid = VolumeGrid.cube(n, vox)
    truth = PH.voxelize(grid, PH.random_ellipsoids(seed, 10), device=f"cuda:{device}")
    plan = JosephPlan(scan.views(), det, det, grid, device=device)
    truth *= 3.0 / float(plan.forward(truth).max())
    b = plan.forward(truth)
    PH.poisson_noise_(b, i0, seed=seed + 1)
    return scan, grid, plan, truth, b


def rel_rmse(x: torch.Tensor, truth: torch.Tensor) -> float:
    return float(torch.sqrt(((x - truth).double() ** 2).mean()) /
                 torch.sqrt((truth.double() ** 2).mean()))


def _main():
    import argparse
    import json
    import time

    from .geometry import RampFilter
    from .projectors import FdkPlan
    ap = argparse.ArgumentParser(description="TV-regularised unrolled reconstruction vs CGLS and FDK")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--views", type=int, default=90)
    ap.add_argument("--det", type=int, default=384)
    ap.add_argument("--vox", type=float, default=0.5)
    ap.add_argument("--pix", type=float, default=0.8)
    ap.add_argument("--adam-steps", type=int, default=50)
    ap.add_argument("--unrolled", type=int, default=10)
    ap.add_argument("--tv", type=float, default=1e-3)
    ap.add_argument("--i0", type=float, default=5e4)
    ap.add_argument("--cgls-iters", type=int, default=50)
    ap.add_argument("--init", choices=["zero", "fdk"], default="fdk",
                    help="start of the unrolled iterations: zeros or the FDK reconstruction")
    ap.add_argument("--no-momentum", action="store_true", help="plain gradient steps")
    ap.add_argument("--lr-rel", type=float, default=0.01)
    a = ap.parse_args()
    torch.cuda.set_device(0)
    scan, grid, plan, truth, b = make_problem(a.n, a.views, a.det, a.vox, a.pix, a.i0)
    torch.cuda.synchronize()
    out = {"workload": f"tv-{a.n}^3-{a.views}v-{a.det}^2", "adam_steps": a.adam_steps,
           "unrolled": a.unrolled, "tv_weight": a.tv, "noise_i0": a.i0,
           "objective": "1/2 mean((Ax-b)^2) + tv mean(sqrt(|grad x|^2 + 1e-8))"}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    op = JosephProjector(plan)
    ev0.record()
    xc, norms = cgls(plan, b, a.cgls_iters)
    ev1.record()
    torch.cuda.synchronize()
    out["cgls"] = {"iters": a.cgls_iters, "ms": ev0.elapsed_time(ev1),
                   "rel_rmse_vs_phantom": rel_rmse(xc, truth),
                   "objective": float(objective(op, xc, b, a.tv))}
    fdk = FdkPlan(scan.views(), a.det, a.det, scan.scan_range, grid, RampFilter.named("shepplogan"))
    xf = fdk.execute(b)
    fdk.close()
    out["fdk"] = {"rel_rmse_vs_phantom": rel_rmse(xf, truth)}
    torch.cuda.reset_peak_memory_stats()
    ev0.record()
    t0 = time.perf_counter()
    xt, model, losses = unrolled_tv(plan, b, a.adam_steps, a.unrolled, a.tv, lr_rel=a.lr_rel,
                                    x_init=xf if a.init == "fdk" else None,
                                    momentum=not a.no_momentum)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    out["unrolled_tv"] = {"ms": ms, "ms_per_adam_step": ms / a.adam_steps,
                          "wall_s": time.perf_counter() - t0,
                          "rel_rmse_vs_phantom": rel_rmse(xt, truth),
                          "objective": float(objective(op, xt, b, a.tv)),
                          "objective_first": losses[0], "objective_last_step": losses[-1],
                          "peak_mem_gb": torch.cuda.max_memory_allocated() / 1e9,
                          "alphas": [float(v) for v in torch.exp(model.log_alpha.detach()).cpu()]}
    out["unrolled_tv"].update(init=a.init, momentum=not a.no_momentum, lr_rel=a.lr_rel)
    plan.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    _main()
