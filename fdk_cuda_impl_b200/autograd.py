"""Differentiable Joseph projection: torch.autograd.Function over the C-ABI.

forward:  y = A x   (ykb_joseph_fp)
backward: dx = A^T dy (ykb_joseph_bp, the exact transpose of the same
discrete weights), so gradients of any loss of A x are exact up to FP32
accumulation rounding.
"""
from __future__ import annotations

import torch

from .projectors import JosephPlan


class JosephProjectFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume: torch.Tensor, plan: JosephPlan) -> torch.Tensor:
        ctx.plan = plan
        return plan.forward(volume.contiguous())

    @staticmethod
    def backward(ctx, grad_proj: torch.Tensor):
        return ctx.plan.adjoint(grad_proj.contiguous()), None


class JosephBackprojectFn(torch.autograd.Function):
    """x = A^T y with gradient A dx (the adjoint as a differentiable op)."""

    @staticmethod
    def forward(ctx, proj: torch.Tensor, plan: JosephPlan) -> torch.Tensor:
        ctx.plan = plan
        return plan.adjoint(proj.contiguous())

    @staticmethod
    def backward(ctx, grad_vol: torch.Tensor):
        return ctx.plan.forward(grad_vol.contiguous()), None


class JosephProjector(torch.nn.Module):
    """nn.Module wrapper: forward(volume) -> projections (differentiable)."""

    def __init__(self, plan: JosephPlan):
        super().__init__()
        self.plan = plan

    def forward(self, volume: torch.Tensor) -> torch.Tensor:
        return JosephProjectFn.apply(volume, self.plan)

    def adjoint(self, proj: torch.Tensor) -> torch.Tensor:
        return JosephBackprojectFn.apply(proj, self.plan)


def project(volume: torch.Tensor, plan: JosephPlan) -> torch.Tensor:
    return JosephProjectFn.apply(volume, plan)


def backproject(proj: torch.Tensor, plan: JosephPlan) -> torch.Tensor:
    return JosephBackprojectFn.apply(proj, plan)
