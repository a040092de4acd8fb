"""Differentiable ray cast: a ``torch.autograd.Function`` over the C ABI.

The brick pool is a float32 CUDA tensor of shape ``(slots, 1000, 4)`` (RGBA
per texel, brick-linear 10x10x10 slots, the layout of ``vv_brickpool_*``)
attached to a :class:`~voxviz_b200.Context` as caller-owned memory.  The
forward runs the checkpointing ray cast of every view
(``vv_render_forward_ckpt``: the same colour as ``vv_render``, bit for bit);
the backward runs the adjoint (``vv_backward_ex``), which adds dL/d(texel)
into a zeroed tensor of the pool's shape; with ``spread`` the views' atomics
go to four copies of the gradient in context memory (three times the pool's
size; fewer concurrent atomics on one texel), added into the tensor once
after the last view - a pass over the whole pool, which on dense pools of
many slots costs more than the contention it removes (the default is off).  The forward's control flow (descent,
step counts, early termination) is held fixed, as for any reverse-mode
derivative of the shader (GigaVoxelsNoLighting.frag:280,354 composite
``dst += (1 - dst.a) * src``).

Work is ordered on torch's current stream: the context is pointed at it
before every launch, so no extra synchronisation is needed around the calls.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from . import Context, Uniforms

DEFAULT_PER_RAY = 16


class _DeviceBytes:
    """A borrowed device range exposed through ``__cuda_array_interface__``."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def pool_tensor_from_context(ctx: Context, device: torch.device | None = None) -> torch.Tensor:
    """A torch-owned float32 copy ``(slots, 1000, 4)`` of the context's FP32 brick pool."""
    from . import VV_FMT_FP32
    if ctx.fmt != VV_FMT_FP32:
        raise ValueError("the differentiable ray cast needs an FP32 brick pool")
    ptr, nbytes = ctx.brickpool_ptr()
    if not ptr:
        raise RuntimeError("the context has no brick pool")
    dev = device or torch.device("cuda", torch.cuda.current_device())
    src = torch.as_tensor(_DeviceBytes(ptr, nbytes), device=dev)
    torch.cuda.current_stream(dev).synchronize()
    sx, sy, sz = ctx.slots
    return src.view(torch.float32).reshape(sx * sy * sz, 1000, 4).clone()


def attach_pool(ctx: Context, pool: torch.Tensor, slots: Sequence[int]) -> None:
    """Make ``pool`` (float32, contiguous, ``(prod(slots), 1000, 4)``) the context's brick pool."""
    if pool.dtype != torch.float32 or not pool.is_cuda or not pool.is_contiguous():
        raise ValueError("pool must be a contiguous float32 CUDA tensor")
    n = int(slots[0]) * int(slots[1]) * int(slots[2])
    if tuple(pool.shape) != (n, 1000, 4):
        raise ValueError(f"pool shape {tuple(pool.shape)} does not match slots {tuple(slots)}")
    key = (pool.data_ptr(), tuple(int(s) for s in slots))
    if getattr(ctx, "_attached", None) != key:
        ctx.attach_bricks(pool.data_ptr(), slots, "fp32")
        ctx._attached = key


def _bind_stream(ctx: Context, device: torch.device) -> None:
    ctx.set_stream(torch.cuda.current_stream(device).cuda_stream)


class RayCast(torch.autograd.Function):
    """colour (V, H, W, 4) float32 = ray cast of every view over ``pool``."""

    @staticmethod
    def forward(fctx, pool: torch.Tensor, ctx: Context, slots, uniforms: Sequence[Uniforms], per_ray: int,
                spread: bool = False):
        attach_pool(ctx, pool, slots)
        _bind_stream(ctx, pool.device)
        H, W = uniforms[0].height, uniforms[0].width
        if any(u.height != H or u.width != W for u in uniforms):
            raise ValueError("every view of one call must have the same size")
        V = len(uniforms)
        color = torch.empty((V, H, W, 4), dtype=torch.float32, device=pool.device)
        nb = Context.ckpt_bytes(W, H, per_ray)
        ckpt = torch.empty((V, nb), dtype=torch.uint8, device=pool.device)
        for v, u in enumerate(uniforms):
            ctx.forward_ckpt(u, color[v].data_ptr(), ckpt[v].data_ptr(), per_ray)
        fctx.vctx = ctx
        fctx.slots = slots
        fctx.uniforms = list(uniforms)
        fctx.per_ray = per_ray
        fctx.spread = spread
        fctx.save_for_backward(pool, ckpt)
        return color

    @staticmethod
    def backward(fctx, grad_color: torch.Tensor):
        pool, ckpt = fctx.saved_tensors
        ctx = fctx.vctx
        attach_pool(ctx, pool, fctx.slots)
        _bind_stream(ctx, pool.device)
        g = grad_color.contiguous().to(torch.float32)
        grad = torch.zeros_like(pool)
        last = len(fctx.uniforms) - 1
        for v, u in enumerate(fctx.uniforms):
            ctx.backward_ex(u, g[v].data_ptr(), ckpt[v].data_ptr(), fctx.per_ray, grad.data_ptr(),
                            spread=fctx.spread, keep=fctx.spread and v < last)
        return grad, None, None, None, None, None


def render(pool: torch.Tensor, ctx: Context, slots, uniforms: Sequence[Uniforms],
           per_ray: int = DEFAULT_PER_RAY, spread: bool = False) -> torch.Tensor:
    """Differentiable colour of every view; ``pool`` may require grad."""
    return RayCast.apply(pool, ctx, slots, list(uniforms), per_ray, spread)


def check_status(ctx: Context) -> int:
    """Synchronise and return (and clear) the device status word (0 = fine)."""
    ctx.synchronize()
    return ctx.device_status(clear=True)


def texel_voxel_index(slots: Sequence[int], slot: np.ndarray, texel: np.ndarray) -> np.ndarray:
    """Global pool-texture coordinates (x, y, z) of texel ``texel`` of slot ``slot``."""
    sx, sy = int(slots[0]), int(slots[1])
    s = np.asarray(slot, dtype=np.int64)
    t = np.asarray(texel, dtype=np.int64)
    return np.stack([(s % sx) * 10 + t % 10, ((s // sx) % sy) * 10 + (t // 10) % 10,
                     (s // (sx * sy)) * 10 + t // 100], axis=-1)
