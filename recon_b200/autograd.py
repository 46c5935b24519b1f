"""torch.autograd binding of the EXACT projector pair (a thin test binding).

The EXACT forward and back projectors are exact transposes (every (ray, voxel)
pair carries the same FP32 length in both), so the back projector is the
forward projector's gradient and vice versa.

:func:`mlem_unrolled` runs relaxed MLEM,
    f_{k+1} = f_k * (1 - w + w * A^T(g / A f_k) / s),   s = A^T 1,
which is the reference's update (hf_siddon_recon.hpp:473-474) at w = 1,
differentiably in f_0, g and the scalar relaxation weight w, recomputing each
iteration in the backward pass (torch.utils.checkpoint) so that memory stays
at one image per iteration.
"""
from __future__ import annotations

import torch
from torch.utils.checkpoint import checkpoint

from .api import Plan


class _Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol: torch.Tensor, plan: Plan) -> torch.Tensor:
        ctx.plan = plan
        return plan.fp_views(vol.detach().contiguous())

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        return ctx.plan.bp_views(grad.contiguous()), None


class _Backproject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sino: torch.Tensor, plan: Plan) -> torch.Tensor:
        ctx.plan = plan
        return plan.bp_views(sino.detach().contiguous())

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        return ctx.plan.fp_views(grad.contiguous()), None


def project(vol: torch.Tensor, plan: Plan) -> torch.Tensor:
    """A x for all views of the plan (differentiable)."""
    return _Project.apply(vol, plan)


def backproject(sino: torch.Tensor, plan: Plan) -> torch.Tensor:
    """A^T y (differentiable)."""
    return _Backproject.apply(sino, plan)


def _safe_div(num: torch.Tensor, den: torch.Tensor) -> torch.Tensor:
    # divide1 (hf_cuda_kernels.cuh:370-387): 0 where the denominator is 0,
    # written so that the masked branch carries no inf/NaN gradient
    nz = den != 0
    return torch.where(nz, num / torch.where(nz, den, torch.ones_like(den)), torch.zeros_like(num))


def mlem_step(f: torch.Tensor, g: torch.Tensor, sens: torch.Tensor, w: torch.Tensor, plan: Plan) -> torch.Tensor:
    ratio = _safe_div(g, project(f, plan))
    upd = _safe_div(backproject(ratio, plan), sens)
    return f * (1.0 - w + w * upd)


def mlem_unrolled(plan: Plan, g: torch.Tensor, iters: int, w: torch.Tensor | float = 1.0,
                  f0: torch.Tensor | None = None, use_checkpoint: bool = True) -> torch.Tensor:
    """`iters` relaxed MLEM iterations, differentiable in g, w and f0."""
    if not torch.is_tensor(w):
        w = torch.tensor(float(w), device=g.device)
    sens = plan.sensitivity()
    f = plan.new_volume(1.0) if f0 is None else f0
    for _ in range(iters):
        if use_checkpoint:
            f = checkpoint(mlem_step, f, g, sens, w, plan, use_reentrant=False)
        else:
            f = mlem_step(f, g, sens, w, plan)
    return f
