"""Differentiable rendering: the splatting path behind torch.autograd.Function.

``render(params, camera, background)`` returns an (H, W, 3) image whose backward runs
the CUDA raster backward, the per-Gaussian reduction and the projection / SH VJPs
(msplat_cuda_render_backward) and yields gradients for all six parameter tensors.
``ssim_l1_loss(image, target, ssim_weight)`` is msplat's training loss, L1 +
ssim_weight * (1 - SSIM) (core/cpu/msplat_cpu.cpp:669-785), forward and backward in
one fused kernel. Their composition gives exactly the gradients msplat_train_step
computes before its Adam update.

Per-pixel transmittance is not stored between forward and backward: the backward
recovers it from the final transmittance, back to front, as the reference does
(core/cpu/msplat_cpu.cpp:996-997), so memory does not grow with the number of
(pixel, Gaussian) contributions.

Each forward holds a context (its frame cache) until its backward has run, taken
from a pool, so several renders may be alive in one graph.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import List, Optional

import numpy as np
import torch

from ._lib import check, lib
from .backend import Context, GaussianParams, ptr
from .camera import CameraSetup

_POOL: List[Context] = []
_POOL_LOCK = threading.Lock()
_STORE_T = 0
_CHUNKED = ("off", 512)


def set_transmittance_mode(mode: str = "recompute", capacity: int = 256) -> None:
    """"recompute" (default): the backward recovers each pixel's transmittance from its
    final value by division, back to front, as the reference does; memory does not grow
    with the number of contributions. "store": the forward stores the transmittance
    before each of a pixel's first ``capacity`` contributions (4 bytes each per pixel)
    and the backward reads it (no division; pixels beyond capacity fall back)."""
    global _STORE_T
    if mode not in ("recompute", "store"):
        raise ValueError("mode must be 'recompute' or 'store'")
    _STORE_T = int(capacity) if mode == "store" else 0


def set_chunked_mode(mode: str = "off", chunk_len: int = 512) -> None:
    """Depth-chunked compositing of the renders and their backward (the Metal backend's
    path for small frames): "off" (default, one pass per tile as core/cpu), "auto"
    (frames of fewer than 400 tiles) or "on"; see Context.set_chunked."""
    global _CHUNKED
    if mode not in Context._CHUNK_MODES:
        raise ValueError(f"mode must be one of {sorted(Context._CHUNK_MODES)}")
    _CHUNKED = (mode, int(chunk_len))


def _acquire() -> Context:
    with _POOL_LOCK:
        c = _POOL.pop() if _POOL else None
    if c is None:
        c = Context()
    if c.store_transmittance != _STORE_T:
        c.set_store_transmittance(_STORE_T)
    if (c.chunked, c.chunk_len) != _CHUNKED:
        c.set_chunked(*_CHUNKED)
    return c


def pool_device_bytes() -> int:
    """Device memory held by the idle contexts of the pool."""
    with _POOL_LOCK:
        return sum(c.device_bytes() for c in _POOL)


def _release(c: Context) -> None:
    with _POOL_LOCK:
        _POOL.append(c)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


class _Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, scales, quats, features_dc, features_rest, opacities, setup: CameraSetup, background,
                degrees_to_use: Optional[int], glob_scale: float, clip_thresh: float):
        p = GaussianParams(*[t.detach().contiguous() for t in
                             (means, scales, quats, features_dc, features_rest, opacities)])
        p.validate()
        frame = _acquire()
        img = frame.render(p, setup, background, degrees_to_use, glob_scale, clip_thresh)
        needs = any(ctx.needs_input_grad[:6])
        if needs:
            ctx.frame = frame
            ctx.params = p
            ctx.setup = setup
            ctx.background = _f32(background)
            ctx.dtu = p.sh_degree if degrees_to_use is None else degrees_to_use
            ctx.glob_scale = glob_scale
            ctx.clip = clip_thresh
        else:
            _release(frame)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        frame: Context = ctx.frame
        p: GaussianParams = ctx.params
        cam: CameraSetup = ctx.setup
        try:
            frame.bind_stream()
            g = [torch.empty_like(t) for t in p.tensors()]
            v = grad_img.contiguous().to(torch.float32)
            check(lib().msplat_cuda_render_backward(
                frame.handle, p.n, ptr(p.means), ptr(p.scales), ctx.glob_scale, ptr(p.quats),
                cam.viewmat.ctypes.data, cam.projmat.ctypes.data, cam.fx, cam.fy, cam.cx, cam.cy, cam.height,
                cam.width, cam.tiles_x, cam.tiles_y, ctx.clip, p.sh_degree, ctx.dtu, cam.cam_pos.ctypes.data,
                ctx.background.ctypes.data, ptr(v), *[ptr(t) for t in g]))
        finally:
            _release(frame)
            ctx.frame = None
        return (*g, None, None, None, None, None)


class _SsimL1(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, target, ssim_weight: float):
        img = image.detach().contiguous().to(torch.float32)
        tgt = target.detach().contiguous().to(torch.float32)
        if img.shape != tgt.shape or img.dim() != 3 or img.shape[2] != 3:
            raise ValueError("image and target must both be (H, W, 3)")
        h, w = int(img.shape[0]), int(img.shape[1])
        v = torch.empty_like(img)
        loss = torch.empty((), dtype=torch.float32, device=img.device)
        frame = _acquire()
        try:
            frame.bind_stream()
            check(lib().msplat_cuda_ssim_loss(frame.handle, ptr(img), ptr(tgt), h, w, float(ssim_weight),
                                              1.0 / (h * w * 3), ptr(v), ptr(loss)))
        finally:
            _release(frame)
        ctx.save_for_backward(v)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        (v,) = ctx.saved_tensors
        return grad_loss * v, None, None


def render(params: GaussianParams, setup: CameraSetup, background, degrees_to_use: Optional[int] = None,
           glob_scale: float = 1.0, clip_thresh: float = 0.01) -> torch.Tensor:
    """Differentiable msplat_render: (H, W, 3) float32 image on the GPU."""
    return _Render.apply(params.means, params.scales, params.quats, params.features_dc, params.features_rest,
                         params.opacities, setup, background, degrees_to_use, glob_scale, clip_thresh)


def ssim_l1_loss(image: torch.Tensor, target: torch.Tensor, ssim_weight: float = 0.2) -> torch.Tensor:
    """msplat's training loss, differentiable in ``image``."""
    return _SsimL1.apply(image, target, ssim_weight)
