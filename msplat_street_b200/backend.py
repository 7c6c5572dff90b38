"""Torch-facing wrapper of the C-ABI: contexts, render, train step, frame access.

Device memory comes from torch (CUDA tensors); the kernels run on the context's
stream, which is bound to torch's current stream at each call so torch and the
library order their work on one queue.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from .camera import CameraSetup
from ._lib import check, lib

PARAM_NAMES = ("means", "scales", "quats", "features_dc", "features_rest", "opacities")
_FRAME_INT = {"radii", "tile_start", "tile_end", "isect_gid", "final_idx"}


def ptr(t: Optional[torch.Tensor]):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor (got {t.dtype} on {t.device})")


@dataclass
class GaussianParams:
    """The six trainable arrays, float32 CUDA tensors in bindings.h layouts."""

    means: torch.Tensor
    scales: torch.Tensor
    quats: torch.Tensor
    features_dc: torch.Tensor
    features_rest: torch.Tensor
    opacities: torch.Tensor

    @classmethod
    def from_numpy(cls, g, device="cuda") -> "GaussianParams":
        return cls(*[torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device) for a in g.arrays()])

    def tensors(self) -> List[torch.Tensor]:
        return [self.means, self.scales, self.quats, self.features_dc, self.features_rest, self.opacities]

    @property
    def n(self) -> int:
        return int(self.means.shape[0])

    @property
    def sh_degree(self) -> int:
        b = self.features_rest.shape[1] + 1 if self.features_rest.dim() == 3 else 1
        return 0 if b <= 1 else 1 if b <= 4 else 2 if b <= 9 else 3 if b <= 16 else 4

    def clone(self) -> "GaussianParams":
        return GaussianParams(*[t.clone() for t in self.tensors()])

    def numpy(self):
        return [t.detach().cpu().numpy() for t in self.tensors()]

    def validate(self) -> None:
        for nm, t in zip(PARAM_NAMES, self.tensors()):
            require_cuda(t, nm)
        n = self.n
        shapes = [(n, 3), (n, 3), (n, 4), (n, 3), None, (n, 1)]
        for nm, t, s in zip(PARAM_NAMES, self.tensors(), shapes):
            if s is not None and tuple(t.shape) != s and not (nm == "opacities" and tuple(t.shape) == (n,)):
                raise ValueError(f"{nm} has shape {tuple(t.shape)}, expected {s}")
        if self.features_rest.shape[0] != n:
            raise ValueError("features_rest must have N rows")


@dataclass
class AdamState:
    """First and second moments for the six groups plus the hyper-parameters."""

    exp_avg: List[torch.Tensor]
    exp_avg_sq: List[torch.Tensor]
    lrs: List[float]
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    step: int = 0

    @classmethod
    def zeros_like(cls, p: GaussianParams, lrs) -> "AdamState":
        return cls([torch.zeros_like(t) for t in p.tensors()], [torch.zeros_like(t) for t in p.tensors()], list(lrs))

    def step_scalars(self):
        """Model::fullIteration's bias-corrected step sizes (core/src/model.cpp:638-651)."""
        bc1 = np.float32(1.0) - np.float32(self.beta1) ** np.float32(self.step)
        bc2 = np.float32(1.0) - np.float32(self.beta2) ** np.float32(self.step)
        ss = _f32([np.float32(lr) / bc1 for lr in self.lrs])
        b2 = _f32([np.sqrt(bc2)] * 6)
        return ss, b2


class Context:
    """One msplat_cuda context: a frame cache plus the stream it works on."""

    def __init__(self, keep_grads: bool = False):
        if not torch.cuda.is_available():
            raise _lib.MsplatCudaError("msplat_street_b200 needs a CUDA device (no CPU fallback)")
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.msplat_cuda_ctx_create(C.byref(h)))
        self.handle = h
        self.keep_grads = keep_grads
        if keep_grads:
            check(self._lib.msplat_cuda_ctx_set_option(h, b"keep_grads", 1))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.msplat_cuda_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bind_stream(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        s = stream if stream is not None else torch.cuda.current_stream()
        check(self._lib.msplat_cuda_ctx_set_stream(self.handle, C.c_void_p(s.cuda_stream)))

    # -- bindings.h:81-91 ------------------------------------------------------------
    def render_raw(self, p: GaussianParams, cam: CameraSetup, background, degrees_to_use: Optional[int] = None,
                   glob_scale: float = 1.0, clip_thresh: float = 0.01):
        """msplat_render; returns the device pointer of the cached (H, W, 3) image."""
        self.bind_stream()
        deg = p.sh_degree
        dtu = deg if degrees_to_use is None else degrees_to_use
        bg = _f32(background)
        out = C.c_void_p()
        check(self._lib.msplat_cuda_render(
            self.handle, p.n, ptr(p.means), ptr(p.scales), glob_scale, ptr(p.quats), cam.viewmat.ctypes.data,
            cam.projmat.ctypes.data, cam.fx, cam.fy, cam.cx, cam.cy, cam.height, cam.width, cam.tiles_x,
            cam.tiles_y, clip_thresh, deg, dtu, cam.cam_pos.ctypes.data, ptr(p.features_dc), ptr(p.features_rest),
            ptr(p.opacities), bg.ctypes.data, C.byref(out)))
        return out.value

    def render(self, p: GaussianParams, cam: CameraSetup, background, degrees_to_use=None, glob_scale=1.0,
               clip_thresh=0.01, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """msplat_render, copied out of the frame cache into a torch tensor."""
        src = self.render_raw(p, cam, background, degrees_to_use, glob_scale, clip_thresh)
        if out is None:
            out = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device=p.means.device)
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out), C.c_void_p(src), out.numel() * 4))
        return out

    # -- bindings.h:100-118 ----------------------------------------------------------
    def train_step(self, p: GaussianParams, adam: AdamState, cam: CameraSetup, background, gt: torch.Tensor,
                   stats=None, ssim_weight: float = 0.2, degrees_to_use: Optional[int] = None,
                   glob_scale: float = 1.0, clip_thresh: float = 0.01, sync_loss: bool = False,
                   num_adam_groups: int = 6):
        """msplat_train_step. ``adam.step`` is advanced first (as Model::fullIteration
        does). Returns the loss as a float when ``sync_loss`` else None (the loss stays
        on the device, see ``loss_tensor``)."""
        self.bind_stream()
        deg = p.sh_degree
        dtu = deg if degrees_to_use is None else degrees_to_use
        require_cuda(gt, "gt")
        adam.step += 1
        ss, bc2 = adam.step_scalars()
        m1 = (C.c_void_p * 6)(*[t.data_ptr() for t in adam.exp_avg])
        m2 = (C.c_void_p * 6)(*[t.data_ptr() for t in adam.exp_avg_sq])
        bg = _f32(background)
        vis, gn, ms = (stats if stats is not None else (None, None, None))
        loss = C.c_float(0.0)
        check(self._lib.msplat_cuda_train_step(
            self.handle, p.n, ptr(p.means), ptr(p.scales), glob_scale, ptr(p.quats), cam.viewmat.ctypes.data,
            cam.projmat.ctypes.data, cam.fx, cam.fy, cam.cx, cam.cy, cam.height, cam.width, cam.tiles_x,
            cam.tiles_y, clip_thresh, deg, dtu, cam.cam_pos.ctypes.data, ptr(p.features_dc), ptr(p.features_rest),
            ptr(p.opacities), bg.ctypes.data, ptr(gt), ssim_weight, 1.0 / (cam.width * cam.height * 3),
            num_adam_groups, C.cast(m1, C.c_void_p), C.cast(m2, C.c_void_p), ss.ctypes.data, bc2.ctypes.data,
            adam.beta1, adam.beta2, adam.eps, ptr(vis), ptr(gn), ptr(ms), 1.0 / max(cam.width, cam.height), None,
            C.byref(loss) if sync_loss else None))
        return float(loss.value) if sync_loss else None

    def loss_tensor(self) -> torch.Tensor:
        """The last train step's loss as a 0-d CUDA tensor (copied, no host sync)."""
        src = C.c_void_p()
        check(self._lib.msplat_cuda_loss_device(self.handle, C.byref(src)))
        out = torch.empty((), dtype=torch.float32, device="cuda")
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out), src, 4))
        return out

    # -- intermediates -------------------------------------------------------------
    def frame(self, name: str) -> torch.Tensor:
        """A copy of one frame-cache buffer (see msplat_cuda_frame)."""
        src = C.c_void_p()
        cnt = C.c_int64()
        check(self._lib.msplat_cuda_frame(self.handle, name.encode(), C.byref(src), C.byref(cnt)))
        dt = torch.int32 if name in _FRAME_INT else torch.float32
        out = torch.empty(int(cnt.value), dtype=dt, device="cuda")
        if cnt.value:
            check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out), src, int(cnt.value) * 4))
        return out

    def num_isects(self) -> int:
        return int(self._lib.msplat_cuda_num_isects(self.handle))

    def sync(self) -> None:
        check(self._lib.msplat_cuda_sync(self.handle))

    def cleanup(self) -> None:
        check(self._lib.msplat_cuda_cleanup(self.handle))
