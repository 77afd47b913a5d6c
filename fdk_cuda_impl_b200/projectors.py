"""Torch-facing plans over the libykb C-ABI.

FdkPlan    -- cosine preweight + ramp filter + weighted backprojection
JosephPlan -- Joseph forward projector A and its exact transpose A^T

Tensors stay on the GPU; every call is ordered on the current torch CUDA
stream of the plan's device.  There is no CPU path: all compute runs in
libykb.so's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .geometry import RampFilter, VolumeGrid


def _stream_handle(device: int) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _check_tensor(t: torch.Tensor, shape, dtypes, device: int, what: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA tensor")
    if t.device.index != device:
        raise ValueError(f"{what} lives on cuda:{t.device.index}, the plan on cuda:{device}")
    if t.dtype not in dtypes:
        raise TypeError(f"{what} dtype {t.dtype} not in {dtypes}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what} shape {tuple(t.shape)} != {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")


def _dtype_code(t: torch.Tensor) -> int:
    return L.DTYPE_BF16 if t.dtype == torch.bfloat16 else L.DTYPE_F32


PARKER_MODES = {"auto": 0, "disabled": 1, "enabled": 2}


class FdkPlan:
    """FDK for a fixed view sequence (ykb_fdk_plan_create_ex).

    parker: None (no short-scan weighting) or "auto" / "enabled" / "disabled"
    (YK::EParkerMode); the short-scan weights measure each view's position
    from start_angle_rad in rotation_direction (+1/-1)."""

    def __init__(self, views: np.ndarray, nu: int, nv: int, scan_range: float,
                 grid: VolumeGrid, filt: RampFilter | None = None, precision: str = "fp32",
                 device: int = 0, parker: str | None = None, start_angle_rad: float = 0.0,
                 rotation_direction: int = 1):
        self.lib = L.load()
        self.views = np.ascontiguousarray(views, dtype=L.VIEW_DTYPE)
        self.nu, self.nv, self.grid, self.device = nu, nv, grid, device
        self.filt = filt or RampFilter()
        self.precision = {"fp32": L.PRECISION_FP32, "bf16": L.PRECISION_BF16}[precision]
        self._vol = grid.struct()
        self._flt = self.filt.struct()
        h = C.c_void_p()
        mode = PARKER_MODES["disabled" if parker is None else parker]
        L.check(self.lib.ykb_fdk_plan_create_ex(L.views_ptr(self.views), len(self.views), nu, nv,
                                                scan_range, start_angle_rad, rotation_direction,
                                                C.byref(self._vol), C.byref(self._flt),
                                                self.precision, mode, device, C.byref(h)))
        self._h = h

    @property
    def n_views(self) -> int:
        return len(self.views)

    @property
    def filtered_dtype(self):
        return torch.float32

    def workspace_bytes(self) -> int:
        return int(self.lib.ykb_fdk_workspace_bytes(self._h))

    def check(self) -> None:
        """Synchronises the current stream and raises on a device-side error."""
        L.check(self.lib.ykb_fdk_check(self._h, _stream_handle(self.device)))

    def stage_timing(self, enable: bool = True) -> None:
        """Records CUDA events around each filter and backprojection launch
        group of later calls (ykb_fdk_stage_timing)."""
        L.check(self.lib.ykb_fdk_stage_timing(self._h, 1 if enable else 0))

    def stage_times(self) -> dict:
        """Summed device times (ms) and launch-group counts of each stage since
        the last call; synchronises the current stream."""
        fm, bm = C.c_double(0.0), C.c_double(0.0)
        fg, bg = C.c_int(0), C.c_int(0)
        L.check(self.lib.ykb_fdk_stage_times(self._h, _stream_handle(self.device), C.byref(fm),
                                             C.byref(fg), C.byref(bm), C.byref(bg)))
        return {"filter_ms": fm.value, "filter_groups": fg.value,
                "backproject_ms": bm.value, "backproject_groups": bg.value}

    def _vol_out(self, volume):
        if volume is None:
            return torch.empty(self.grid.shape, dtype=torch.float32, device=f"cuda:{self.device}")
        _check_tensor(volume, self.grid.shape, (torch.float32,), self.device, "volume")
        return volume

    def execute(self, proj: torch.Tensor, volume: torch.Tensor | None = None, view_offset: int = 0,
                clear: bool = True) -> torch.Tensor:
        """Reconstructs (or accumulates) views [view_offset, view_offset+len(proj))."""
        n = proj.shape[0]
        _check_tensor(proj, (n, self.nv, self.nu), (torch.float32, torch.bfloat16), self.device,
                      "projections")
        volume = self._vol_out(volume)
        L.check(self.lib.ykb_fdk_execute(self._h, C.c_void_p(proj.data_ptr()), _dtype_code(proj),
                                         view_offset, n, C.c_void_p(volume.data_ptr()),
                                         1 if clear else 0, _stream_handle(self.device)))
        return volume

    def execute_host(self, proj: torch.Tensor, volume: torch.Tensor | None = None,
                     view_offset: int = 0, clear: bool = True,
                     host_out: torch.Tensor | None = None) -> torch.Tensor:
        """FDK of projections held in host memory (pin them for copy/compute
        overlap): batches stream to the device while earlier ones are filtered
        and backprojected.  With host_out (a contiguous float32 host tensor,
        pinned for overlap) the volume is also copied there, slab by slab
        behind the last batch's kernels (ykb_fdk_execute_host_out).
        Asynchronous on the current stream; `proj` and `host_out` must stay
        alive until that stream has run the work."""
        n = proj.shape[0]
        if proj.device.type != "cpu" or not proj.is_contiguous():
            raise ValueError("projections must be a contiguous host tensor")
        if tuple(proj.shape) != (n, self.nv, self.nu) or proj.dtype not in (torch.float32,
                                                                              torch.bfloat16):
            raise ValueError(f"projections must be float32/bfloat16 [n][{self.nv}][{self.nu}]")
        volume = self._vol_out(volume)
        if host_out is None:
            L.check(self.lib.ykb_fdk_execute_host(self._h, C.c_void_p(proj.data_ptr()),
                                                  _dtype_code(proj), view_offset, n,
                                                  C.c_void_p(volume.data_ptr()), 1 if clear else 0,
                                                  _stream_handle(self.device)))
            return volume
        if (host_out.device.type != "cpu" or not host_out.is_contiguous() or
                host_out.dtype != torch.float32 or tuple(host_out.shape) != tuple(self.grid.shape)):
            raise ValueError(f"host_out must be a contiguous float32 host tensor {self.grid.shape}")
        L.check(self.lib.ykb_fdk_execute_host_out(self._h, C.c_void_p(proj.data_ptr()),
                                                  _dtype_code(proj), view_offset, n,
                                                  C.c_void_p(volume.data_ptr()),
                                                  C.c_void_p(host_out.data_ptr()),
                                                  1 if clear else 0, _stream_handle(self.device)))
        return volume

    def filter(self, proj: torch.Tensor, view_offset: int = 0) -> torch.Tensor:
        n = proj.shape[0]
        _check_tensor(proj, (n, self.nv, self.nu), (torch.float32, torch.bfloat16), self.device,
                      "projections")
        out = torch.empty((n, self.nv, self.nu), dtype=self.filtered_dtype, device=proj.device)
        L.check(self.lib.ykb_fdk_filter(self._h, C.c_void_p(proj.data_ptr()), _dtype_code(proj),
                                        view_offset, n, C.c_void_p(out.data_ptr()),
                                        _stream_handle(self.device)))
        return out

    def backproject(self, filtered: torch.Tensor, volume: torch.Tensor | None = None,
                    view_offset: int = 0, clear: bool = True) -> torch.Tensor:
        n = filtered.shape[0]
        _check_tensor(filtered, (n, self.nv, self.nu), (torch.float32, torch.bfloat16),
                      self.device, "filtered projections")
        volume = self._vol_out(volume)
        L.check(self.lib.ykb_fdk_backproject(self._h, C.c_void_p(filtered.data_ptr()),
                                             _dtype_code(filtered), view_offset, n,
                                             C.c_void_p(volume.data_ptr()), 1 if clear else 0,
                                             _stream_handle(self.device)))
        return volume

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.ykb_fdk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class JosephPlan:
    """Joseph projector pair for a fixed view sequence (ykb_joseph_plan_create)."""

    def __init__(self, views: np.ndarray, nu: int, nv: int, grid: VolumeGrid, device: int = 0):
        self.lib = L.load()
        self.views = np.ascontiguousarray(views, dtype=L.VIEW_DTYPE)
        self.nu, self.nv, self.grid, self.device = nu, nv, grid, device
        self._vol = grid.struct()
        h = C.c_void_p()
        L.check(self.lib.ykb_joseph_plan_create(L.views_ptr(self.views), len(self.views), nu, nv,
                                                C.byref(self._vol), device, C.byref(h)))
        self._h = h

    @property
    def proj_shape(self):
        return (len(self.views), self.nv, self.nu)

    def workspace_bytes(self) -> int:
        return int(self.lib.ykb_joseph_workspace_bytes(self._h))

    def forward(self, volume: torch.Tensor, out: torch.Tensor | None = None,
                accumulate: bool = False) -> torch.Tensor:
        _check_tensor(volume, self.grid.shape, (torch.float32,), self.device, "volume")
        if out is None:
            out = torch.empty(self.proj_shape, dtype=torch.float32, device=volume.device)
            accumulate = False
        _check_tensor(out, self.proj_shape, (torch.float32,), self.device, "projections")
        L.check(self.lib.ykb_joseph_fp(self._h, C.c_void_p(volume.data_ptr()),
                                       C.c_void_p(out.data_ptr()), 1 if accumulate else 0,
                                       _stream_handle(self.device)))
        return out

    def adjoint(self, proj: torch.Tensor, out: torch.Tensor | None = None,
                accumulate: bool = False) -> torch.Tensor:
        _check_tensor(proj, self.proj_shape, (torch.float32,), self.device, "projections")
        if out is None:
            out = torch.empty(self.grid.shape, dtype=torch.float32, device=proj.device)
            accumulate = False
        _check_tensor(out, self.grid.shape, (torch.float32,), self.device, "volume")
        L.check(self.lib.ykb_joseph_bp(self._h, C.c_void_p(proj.data_ptr()),
                                       C.c_void_p(out.data_ptr()), 1 if accumulate else 0,
                                       _stream_handle(self.device)))
        return out

    def backproject_pseudo(self, proj: torch.Tensor, out: torch.Tensor | None = None,
                           accumulate: bool = False) -> torch.Tensor:
        """BP_FDK_PseudoMatched: voxel-driven bilinear backprojection with the
        weight L^3 / (|P - S|^2 SDD_plane) x voxel volume / pixel area, an
        approximate transpose of the forward projector
        (src/FlatFpBp/BP/kernels/YkBpFdkKernel.cu:356-450)."""
        return self.apply(L.TASK_BP_FDK_PSEUDO_MATCHED, proj, out, accumulate)

    def forward_siddon(self, volume: torch.Tensor, out: torch.Tensor | None = None,
                       accumulate: bool = False) -> torch.Tensor:
        """FP_Siddon: exact voxel intersection lengths of each source-to-pixel
        ray (src/FlatFpBp/FP/kernels/YkFPSiddonKernel.cu:19-129)."""
        return self.apply(L.TASK_FP_SIDDON, volume, out, accumulate)

    def backproject_siddon(self, proj: torch.Tensor, out: torch.Tensor | None = None,
                           accumulate: bool = False) -> torch.Tensor:
        """BP_Siddon_RayDriven: the exact transpose of forward_siddon
        (src/FlatFpBp/BP/kernels/YkBPSiddonKernel.cu:31-127), summed with
        atomics (last bits vary between runs)."""
        return self.apply(L.TASK_BP_SIDDON_RAY_DRIVEN, proj, out, accumulate)

    def apply(self, task: int, x: torch.Tensor, out: torch.Tensor | None = None,
              accumulate: bool = False) -> torch.Tensor:
        """One operator task (ykb_operator_apply; task values of YK::ETask)."""
        forward = task in (L.TASK_FP_JOSEPH, L.TASK_FP_SIDDON)
        in_shape, out_shape = ((self.grid.shape, self.proj_shape) if forward
                               else (self.proj_shape, self.grid.shape))
        _check_tensor(x, in_shape, (torch.float32,), self.device, "input")
        if out is None:
            out = torch.empty(out_shape, dtype=torch.float32, device=x.device)
            accumulate = False
        _check_tensor(out, out_shape, (torch.float32,), self.device, "output")
        L.check(self.lib.ykb_operator_apply(self._h, task, C.c_void_p(x.data_ptr()),
                                            C.c_void_p(out.data_ptr()), 1 if accumulate else 0,
                                            _stream_handle(self.device)))
        return out

    def check(self) -> None:
        """Raises when the device error word of the plan is set."""
        L.check(self.lib.ykb_joseph_check(self._h, _stream_handle(self.device)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.ykb_joseph_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
