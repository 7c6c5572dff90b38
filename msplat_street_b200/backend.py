"""Torch-facing wrapper of the C-ABI: contexts, render, train step, frame access.

Device memory comes from torch (CUDA tensors); the kernels run on the context's
stream, which is bound to torch's current stream at each call so torch and the
library order their work on one queue.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .camera import CameraSetup, logf
from ._lib import check, lib

PARAM_NAMES = ("means", "scales", "quats", "features_dc", "features_rest", "opacities")
_FRAME_INT = {"radii", "tile_start", "tile_end", "isect_gid", "final_idx", "chunk_first", "knn_evals"}


def ptr(t: Optional[torch.Tensor]):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


def _addr(t: Optional[torch.Tensor]):
    return t.data_ptr() if t is not None else None


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
        return adam_step_scalars(self.lrs, self.step, self.beta1, self.beta2)


def adam_step_scalars(lrs, step: int, beta1: float = 0.9, beta2: float = 0.999):
    """Model::fullIteration's bias-corrected Adam scalars (core/src/model.cpp:638-651):
    bc = 1 - pow(beta, t) is evaluated in double (std::pow(float, int)) and stored as
    float; step_size = lr / bc1 and bc2_sqrt = sqrt(bc2) in float."""
    bc1 = np.float32(1.0 - float(np.float32(beta1)) ** int(step))
    bc2 = np.float32(1.0 - float(np.float32(beta2)) ** int(step))
    ss = _f32([np.float32(lr) / bc1 for lr in lrs])
    b2 = _f32([np.sqrt(bc2)] * len(lrs))
    return ss, b2


@dataclass
class BatchItem:
    """One view of a batched render: a scene, a camera and the render scalars."""
    params: "GaussianParams"
    camera: CameraSetup
    background: object
    degrees_to_use: Optional[int] = None
    glob_scale: float = 1.0
    clip_thresh: float = 0.01


_PRIOR_TENSORS = {"sky_tex": torch.float32, "sky_grad": torch.float32, "sky_exp_avg": torch.float32,
                  "sky_exp_avg_sq": torch.float32, "prior_depth": torch.float32, "prior_aux": torch.uint8,
                  "loss_terms": torch.float32, "expo_params": torch.float32, "expo_exp_avg": torch.float32,
                  "expo_exp_avg_sq": torch.float32, "expo_grad": torch.float32}


@dataclass
class PriorStep:
    """Prior-guided extras of a render / train step (core/metal/bindings.h:43-77), over
    CUDA tensors the step reads and, for the trained ones, updates in place: the
    learned sky (texture, gradient, Adam moments), the loss terms and the exposure
    parameters, moments and gradient. Defaults are the reference's."""
    aux: bool = False
    sky: bool = False
    sky_tex: Optional[torch.Tensor] = None          # (sky_h, sky_w, 3)
    sky_grad: Optional[torch.Tensor] = None
    sky_exp_avg: Optional[torch.Tensor] = None
    sky_exp_avg_sq: Optional[torch.Tensor] = None
    sky_frame: Sequence[float] = (0.0,) * 9         # up, e1 (azimuth 0), e2 (azimuth 90 degrees)
    sky_step_size: float = 0.0
    sky_bc2_sqrt: float = 1.0
    prior_depth: Optional[torch.Tensor] = None      # (prior_h, prior_w) float32, 0 = invalid
    prior_aux: Optional[torch.Tensor] = None        # (prior_h, prior_w, 4) uint8: confidence, sky, keep, -
    has_depth: bool = False
    has_sky_mask: bool = False
    depth_weight: float = 0.0
    sky_weight: float = 0.0
    fill_weight: float = 0.0
    huber_delta: float = 0.05
    min_alpha: float = 0.25
    mask_photometric: bool = True
    loss_terms: Optional[torch.Tensor] = None       # [4]: depth, sky, fill, - (zeroed each step)
    exposure: bool = False
    cam_index: int = 0
    expo_params: Optional[torch.Tensor] = None      # (num_cams, 12)
    expo_exp_avg: Optional[torch.Tensor] = None
    expo_exp_avg_sq: Optional[torch.Tensor] = None
    expo_grad: Optional[torch.Tensor] = None        # [12], zeroed after each update
    expo_step_size: float = 0.0
    expo_bc2_sqrt: float = 1.0
    expo_reg: float = 0.0
    log_max_scale_ratio: float = 0.0                # needle cap, <= 0 disables

    def to_c(self) -> "_lib.Prior":
        c = _lib.Prior()
        for name, dt in _PRIOR_TENSORS.items():
            t = getattr(self, name)
            if t is not None and (not t.is_cuda or t.dtype != dt or not t.is_contiguous()):
                raise ValueError(f"PriorStep.{name} must be a contiguous {dt} CUDA tensor")
            setattr(c, name, _addr(t))
        c.aux, c.sky, c.exposure = int(self.aux), int(self.sky), int(self.exposure)
        c.has_depth, c.has_sky_mask = int(self.has_depth), int(self.has_sky_mask)
        c.mask_photometric, c.cam_index = int(self.mask_photometric), int(self.cam_index)
        if self.sky_tex is not None:
            c.sky_h, c.sky_w = int(self.sky_tex.shape[0]), int(self.sky_tex.shape[1])
        if self.prior_depth is not None:
            c.prior_h, c.prior_w = int(self.prior_depth.shape[0]), int(self.prior_depth.shape[1])
        elif self.prior_aux is not None:
            c.prior_h, c.prior_w = int(self.prior_aux.shape[0]), int(self.prior_aux.shape[1])
        if self.expo_params is not None:
            c.expo_num_cams = int(self.expo_params.shape[0])
        c.sky_frame[:] = [float(v) for v in np.asarray(self.sky_frame, np.float32).reshape(9)]
        for name in ("sky_step_size", "sky_bc2_sqrt", "depth_weight", "sky_weight", "fill_weight", "huber_delta",
                     "min_alpha", "expo_step_size", "expo_bc2_sqrt", "expo_reg", "log_max_scale_ratio"):
            setattr(c, name, float(getattr(self, name)))
        return c


class Context:
    """One msplat_cuda context: a frame cache plus the stream it works on."""

    def __init__(self, keep_grads: bool = False, store_transmittance: int = 0, chunked: str = "off",
                 chunk_len: int = 512):
        if not torch.cuda.is_available():
            raise _lib.MsplatCudaError("msplat_street_b200 needs a CUDA device (no CPU fallback)")
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.msplat_cuda_ctx_create(C.byref(h)))
        self.handle = h
        self.raster_variant = 0
        self.raster_shape = 0
        self.keep_grads = keep_grads
        if keep_grads:
            check(self._lib.msplat_cuda_ctx_set_option(h, b"keep_grads", 1))
        self.set_store_transmittance(store_transmittance)
        self.set_chunked(chunked, chunk_len)

    _CHUNK_MODES = {"off": 0, "auto": 1, "on": 2}

    def set_chunked(self, mode: str = "auto", chunk_len: int = 512) -> None:
        """Depth-chunked compositing of single-view frames (the Metal backend's path for
        small frames, core/metal/msplat_metal.metal:2641-3030): "off" composites each
        tile in one pass (core/cpu, the default); "auto" chunks frames of fewer than 400
        tiles, as the Metal backend does (msplat_metal.mm:1101-1117); "on" chunks every
        frame. Frames with a prior always composite in one pass."""
        if mode not in self._CHUNK_MODES:
            raise ValueError(f"chunked must be one of {sorted(self._CHUNK_MODES)}, not {mode!r}")
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"chunk_len", int(chunk_len)))
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"chunked_raster", self._CHUNK_MODES[mode]))
        self.chunked, self.chunk_len = mode, int(chunk_len)

    def set_store_transmittance(self, capacity: int) -> None:
        """0: the backward recovers transmittance by division (the reference's way);
        K > 0: the forward stores it for each pixel's first K contributions."""
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"store_transmittance", int(capacity)))
        self.store_transmittance = int(capacity)

    def device_bytes(self) -> int:
        """Device memory held by this context's caches."""
        return int(self._lib.msplat_cuda_ctx_device_bytes(self.handle))

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

    def render_batch(self, items: Sequence["BatchItem"], outs: Optional[List[torch.Tensor]] = None,
                     stream: Optional[torch.cuda.Stream] = None) -> List[torch.Tensor]:
        """Batched msplat_render (msplat_cuda_render_batch): every item's view rendered
        by one projection, one sort and one persistent rasterizer launch, each image
        equal to the single-view render. Returns (H, W, 3) tensors (``outs`` if given)."""
        self.bind_stream(stream)
        if not items:
            return []
        views = (_lib.View * len(items))()
        res = []
        for k, it in enumerate(items):
            p, cam = it.params, it.camera
            if outs is not None:
                out = outs[k]
                if (out.shape != (cam.height, cam.width, 3) or out.dtype != torch.float32 or not out.is_cuda
                        or not out.is_contiguous()):
                    raise ValueError(f"outs[{k}] must be a contiguous float32 CUDA ({cam.height}, {cam.width}, 3)")
            else:
                out = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device=p.means.device)
            res.append(out)
            w = views[k]
            w.num_points = p.n
            w.means3d, w.scales, w.quats = _addr(p.means), _addr(p.scales), _addr(p.quats)
            w.features_dc, w.features_rest, w.opacities = (_addr(p.features_dc), _addr(p.features_rest),
                                                            _addr(p.opacities))
            w.glob_scale = it.glob_scale
            w.degree = p.sh_degree
            w.degrees_to_use = p.sh_degree if it.degrees_to_use is None else it.degrees_to_use
            w.viewmat[:] = [float(x) for x in cam.viewmat.reshape(-1)]
            w.projmat[:] = [float(x) for x in cam.projmat.reshape(-1)]
            w.fx, w.fy, w.cx, w.cy = cam.fx, cam.fy, cam.cx, cam.cy
            w.img_height, w.img_width = cam.height, cam.width
            w.clip_thresh = it.clip_thresh
            w.cam_pos[:] = [float(x) for x in cam.cam_pos.reshape(-1)]
            w.background[:] = [float(x) for x in _f32(it.background).reshape(-1)]
            w.out_img = out.data_ptr()
        check(self._lib.msplat_cuda_render_batch(self.handle, len(items), views))
        return res

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

    # -- image pipeline, metrics, display (bindings.h:158-180) ------------------------
    def resize_area(self, src: torch.Tensor, out_w: int, out_h: int) -> torch.Tensor:
        """Area resample of an (H, W, 4) uint8 RGBA or (H, W, 3) float32 CUDA image to
        (out_h, out_w, 3) float32."""
        self.bind_stream()
        u8 = src.dtype == torch.uint8
        if not src.is_cuda or not src.is_contiguous() or src.dim() != 3 or src.shape[2] != (4 if u8 else 3) or \
                (not u8 and src.dtype != torch.float32):
            raise ValueError("src must be a contiguous CUDA (H, W, 4) uint8 or (H, W, 3) float32 image")
        out = torch.empty((out_h, out_w, 3), dtype=torch.float32, device=src.device)
        check(self._lib.msplat_cuda_resize_area(self.handle, ptr(src), int(u8), src.shape[1], src.shape[0], ptr(out),
                                                out_w, out_h))
        return out

    def undistort(self, src: torch.Tensor, intr, dist, roi_x: int, roi_y: int, out_w: int,
                  out_h: int) -> torch.Tensor:
        """Brown-Conrady undistortion (intr = fx, fy, cx, cy; dist = k1, k2, p1, p2, k3)
        of an (H, W, 3) float32 image into the (out_h, out_w) crop at (roi_x, roi_y)."""
        self.bind_stream()
        require_cuda(src, "src")
        it, ds = _f32(intr), _f32(dist)
        if it.size != 4 or ds.size != 5:
            raise ValueError("intr needs 4 values and dist 5")
        out = torch.empty((out_h, out_w, 3), dtype=torch.float32, device=src.device)
        check(self._lib.msplat_cuda_undistort(self.handle, ptr(src), src.shape[1], src.shape[0], it.ctypes.data,
                                              ds.ctypes.data, roi_x, roi_y, ptr(out), out_w, out_h))
        return out

    def image_metrics(self, rendered: torch.Tensor, gt: torch.Tensor):
        """(PSNR, SSIM, L1) of two (H, W, 3) float32 CUDA images."""
        self.bind_stream()
        require_cuda(rendered, "rendered")
        require_cuda(gt, "gt")
        if rendered.shape != gt.shape:
            raise ValueError("images differ in shape")
        out = np.zeros(3, np.float64)
        check(self._lib.msplat_cuda_image_metrics(self.handle, ptr(rendered), ptr(gt), rendered.shape[0],
                                                  rendered.shape[1], out.ctypes.data))
        return float(out[0]), float(out[1]), float(out[2])

    def pack_rgba8(self, img: torch.Tensor) -> np.ndarray:
        """(H, W, 3) float32 CUDA image to an (H, W, 4) uint8 host array."""
        self.bind_stream()
        require_cuda(img, "img")
        out = np.empty(tuple(img.shape[:-1]) + (4,), np.uint8)
        check(self._lib.msplat_cuda_pack_rgba8(self.handle, ptr(img), img.numel() // 3, out.ctypes.data))
        return out

    def finalize_depth(self, depth_num: torch.Tensor, final_T: torch.Tensor, inv_scale: float = 1.0):
        """(expected depth, alpha) from the aux render's depth numerator and final T."""
        self.bind_stream()
        require_cuda(depth_num, "depth_num")
        require_cuda(final_T, "final_T")
        d, a = torch.empty_like(depth_num), torch.empty_like(final_T)
        check(self._lib.msplat_cuda_finalize_depth(self.handle, ptr(depth_num), ptr(final_T), depth_num.numel(),
                                                   inv_scale, ptr(d), ptr(a)))
        return d, a

    def set_raster_variant(self, v: int) -> None:
        """Rasterizer staging variant (see raster_variants()); results do not depend on it."""
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"raster_variant", int(v)))
        self.raster_variant = int(v)

    def set_raster_shape(self, s: int) -> None:
        """Block shape of the batched forward rasterizer (see autotune.raster_shapes());
        results do not depend on it."""
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"raster_shape", int(s)))
        self.raster_shape = int(s)

    def set_graph(self, on: bool = True) -> None:
        """Replay a captured CUDA graph of each batched training step (train_batch)."""
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"graph", int(bool(on))))

    def graph_stats(self) -> dict:
        out = (C.c_int64 * 4)()
        check(self._lib.msplat_cuda_train_batch_stats(self.handle, out))
        return {"replays": out[0], "captures": out[1], "overflows": out[2], "isect_capacity": out[3]}

    def train_batch(self, p: GaussianParams, adam: Optional[AdamState], views: Sequence, background,
                    stats=None, ssim_weight: float = 0.2, degrees_to_use: Optional[int] = None,
                    glob_scale: float = 1.0, clip_thresh: float = 0.01, grads: Optional[List[torch.Tensor]] = None,
                    num_adam_groups: int = 6, sync_loss: bool = True):
        """msplat_cuda_train_batch: ``views`` is a sequence of (CameraSetup, target
        tensor) pairs trained in one step (gradients summed, one Adam step when
        ``adam`` is given; ``adam.step`` is advanced first). ``grads`` (6 tensors in
        parameter layout) receives the summed gradients. Returns the per-view losses
        when ``sync_loss``."""
        self.bind_stream()
        deg = p.sh_degree
        dtu = deg if degrees_to_use is None else degrees_to_use
        tv = (_lib.TrainView * len(views))()
        for k, (cam, gt) in enumerate(views):
            require_cuda(gt, f"target {k}")
            if tuple(gt.shape) != (cam.height, cam.width, 3):
                raise ValueError(f"target {k} has shape {tuple(gt.shape)}, camera is {cam.height}x{cam.width}")
            w = tv[k]
            w.viewmat[:] = [float(x) for x in cam.viewmat.reshape(-1)]
            w.projmat[:] = [float(x) for x in cam.projmat.reshape(-1)]
            w.fx, w.fy, w.cx, w.cy = cam.fx, cam.fy, cam.cx, cam.cy
            w.img_height, w.img_width = cam.height, cam.width
            w.cam_pos[:] = [float(x) for x in cam.cam_pos.reshape(-1)]
            w.gt = gt.data_ptr()
        groups = 0
        m1 = m2 = ss = bc2 = None
        if adam is not None:
            groups = num_adam_groups
            adam.step += 1
            s, b = adam.step_scalars()
            ss, bc2 = s.ctypes.data, b.ctypes.data
            m1a = (C.c_void_p * 6)(*[t.data_ptr() for t in adam.exp_avg])
            m2a = (C.c_void_p * 6)(*[t.data_ptr() for t in adam.exp_avg_sq])
            m1, m2 = C.cast(m1a, C.c_void_p), C.cast(m2a, C.c_void_p)
        g = None
        if grads is not None:
            for t, ref in zip(grads, p.tensors()):
                if t.shape != ref.shape:
                    raise ValueError("gradient outputs must match the parameter shapes")
                require_cuda(t, "gradient output")
            ga = (C.c_void_p * 6)(*[t.data_ptr() for t in grads])
            g = C.cast(ga, C.c_void_p)
        vis, gn, ms = (stats if stats is not None else (None, None, None))
        bg = _f32(background)
        losses = np.zeros(len(views), np.float32)
        check(self._lib.msplat_cuda_train_batch(
            self.handle, p.n, ptr(p.means), ptr(p.scales), glob_scale, ptr(p.quats), ptr(p.features_dc),
            ptr(p.features_rest), ptr(p.opacities), deg, dtu, clip_thresh, bg.ctypes.data, len(views), tv,
            ssim_weight, groups, m1, m2, ss, bc2, adam.beta1 if adam else 0.9, adam.beta2 if adam else 0.999,
            adam.eps if adam else 1e-8, ptr(vis), ptr(gn), ptr(ms), g, losses.ctypes.data if sync_loss else None))
        return losses if sync_loss else None

    def loss_tensor(self) -> torch.Tensor:
        """The last train step's loss as a 0-d CUDA tensor (copied, no host sync)."""
        src = C.c_void_p()
        check(self._lib.msplat_cuda_loss_device(self.handle, C.byref(src)))
        out = torch.empty((), dtype=torch.float32, device="cuda")
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out), src, 4))
        return out

    def read_loss_async(self, out: torch.Tensor) -> torch.cuda.Event:
        """Enqueues a copy of the last train step's loss into ``out`` (a one-element
        pinned host float32 tensor) behind the step's kernels and returns an event that
        completes with the copy: the loss is read without stalling the host, so the next
        step can be queued first."""
        if out.is_cuda or out.dtype != torch.float32 or out.numel() < 1 or not out.is_pinned():
            raise ValueError("out must be a pinned host float32 tensor")
        self.bind_stream()
        src = C.c_void_p()
        check(self._lib.msplat_cuda_loss_device(self.handle, C.byref(src)))
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out), src, 4))
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream())
        return ev

    # -- bindings.h:120-155 ----------------------------------------------------------
    def densify(self, n: int, buffers: List[torch.Tensor], exp_avg: List[torch.Tensor],
                exp_avg_sq: List[torch.Tensor], grad_norm: torch.Tensor, vis_counts: torch.Tensor,
                max_2d: torch.Tensor, half_max_dim: float, seed: int, grad_thresh: float = 2e-4,
                size_thresh: float = 0.01, screen_thresh: float = 0.05, check_screen: bool = True,
                cull_alpha: float = 0.1, cull_scale: float = 0.5, cull_screen: float = 0.15,
                check_huge: bool = True) -> int:
        """msplat_densify over capacity-sized buffers (6 params + 12 moments), in place.
        Returns the new Gaussian count (one host synchronisation)."""
        self.bind_stream()
        cap = int(buffers[0].shape[0])
        fr_stride = int(buffers[4].numel() // cap) if cap else 0
        pp = (C.c_void_p * 6)(*[t.data_ptr() for t in buffers])
        m1 = (C.c_void_p * 6)(*[t.data_ptr() for t in exp_avg])
        m2 = (C.c_void_p * 6)(*[t.data_ptr() for t in exp_avg_sq])
        out = C.c_int(0)
        check(self._lib.msplat_cuda_densify(
            self.handle, n, cap, grad_thresh, size_thresh, screen_thresh, int(check_screen), cull_alpha, cull_scale,
            cull_screen, int(check_huge), ptr(grad_norm), ptr(vis_counts), ptr(max_2d), half_max_dim,
            C.cast(pp, C.c_void_p), fr_stride, C.cast(m1, C.c_void_p), C.cast(m2, C.c_void_p),
            C.c_uint32(seed & 0xFFFFFFFF), C.byref(out)))
        return int(out.value)

    def opacity_reset(self, opacities: torch.Tensor, exp_avg: torch.Tensor, exp_avg_sq: torch.Tensor, n: int,
                      reset_logit: float = -1.3862943611198906) -> None:
        self.bind_stream()
        check(self._lib.msplat_cuda_opacity_reset(self.handle, ptr(opacities), ptr(exp_avg), ptr(exp_avg_sq), n,
                                                  reset_logit))

    def radix_sort(self, keys: torch.Tensor, vals: torch.Tensor, key_bits: int) -> None:
        """Stable in-place sort of int64 keys (by their low key_bits) with int32 values."""
        self.bind_stream()
        if keys.dtype != torch.int64 or vals.dtype != torch.int32 or not keys.is_cuda:
            raise ValueError("keys must be int64 and vals int32 CUDA tensors")
        check(self._lib.msplat_cuda_radix_sort(self.handle, ptr(keys), ptr(vals), keys.numel(), key_bits))

    def knn3_mean_dist(self, points: torch.Tensor) -> torch.Tensor:
        self.bind_stream()
        require_cuda(points, "points")
        out = torch.empty(points.shape[0], dtype=torch.float32, device=points.device)
        check(self._lib.msplat_cuda_knn3_mean_dist(self.handle, ptr(points), points.shape[0], ptr(out)))
        return out

    def init_gaussians(self, means: torch.Tensor, rgb: torch.Tensor, seed: int = 42,
                       opacity_logit: Optional[float] = None, sh_degree: int = 3) -> GaussianParams:
        """msplat_init_gaussians + zero SH rest: the Model constructor's start state
        (core/src/model.cpp:57-71). opacity_logit defaults to the constructor's
        std::log(0.1f / 0.9f) (initial opacity 0.1)."""
        self.bind_stream()
        require_cuda(means, "means")
        if opacity_logit is None:
            opacity_logit = float(logf(np.float32(0.1) / np.float32(0.9)))
        n = means.shape[0]
        dev = means.device
        scales = torch.empty((n, 3), dtype=torch.float32, device=dev)
        quats = torch.empty((n, 4), dtype=torch.float32, device=dev)
        dc = torch.empty((n, 3), dtype=torch.float32, device=dev)
        opac = torch.empty((n, 1), dtype=torch.float32, device=dev)
        rgb = rgb.to(device=dev, dtype=torch.uint8).contiguous()
        check(self._lib.msplat_cuda_init_gaussians(self.handle, ptr(means), ptr(rgb), n, seed & 0xFFFFFFFF,
                                                   opacity_logit, ptr(scales), ptr(quats), ptr(dc), ptr(opac)))
        rest = torch.zeros((n, (sh_degree + 1) ** 2 - 1, 3), dtype=torch.float32, device=dev)
        return GaussianParams(means.clone(), scales, quats, dc, rest, opac)

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

    # -- prior-guided extras (bindings.h:43-96) ---------------------------------------
    def set_prior(self, prior: Optional[PriorStep]) -> None:
        """The PriorStep of later render / train_step calls (None: the plain pipeline).
        The tensors must stay alive while it is set; the context keeps a reference."""
        self._prior = prior
        if prior is None:
            check(self._lib.msplat_cuda_set_prior(self.handle, None))
            return
        self._prior_c = prior.to_c()
        check(self._lib.msplat_cuda_set_prior(self.handle, C.byref(self._prior_c)))

    def render_aux_outputs(self):
        """msplat_render_aux_outputs: copies of the expected-depth numerator and the
        final transmittance of the last aux-mode render or step, flat (H * W,)."""
        d, t = C.c_void_p(), C.c_void_p()
        check(self._lib.msplat_cuda_render_aux_outputs(self.handle, C.byref(d), C.byref(t)))
        npix = self.frame("final_Ts").numel()
        out = torch.empty((2, npix), dtype=torch.float32, device="cuda")
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out[0]), d, npix * 4))
        check(self._lib.msplat_cuda_copy_buffer(self.handle, ptr(out[1]), t, npix * 4))
        return out[0], out[1]

    def num_isects(self) -> int:
        return int(self._lib.msplat_cuda_num_isects(self.handle))

    def pair_counts(self):
        """(forward, backward) (pixel, Gaussian) pairs the reference's loops evaluate
        over the last single-view frame (msplat_cuda_frame_pair_counts). Synchronises."""
        out = np.zeros(2, np.int64)
        check(self._lib.msplat_cuda_frame_pair_counts(self.handle, C.c_void_p(out.ctypes.data)))
        return int(out[0]), int(out[1])

    def add_pair_counts(self, acc: torch.Tensor) -> None:
        """Adds the last single-view frame's (forward, backward) pair counts into
        ``acc`` (a CUDA int64 tensor of 2) on the context's stream, without
        synchronising."""
        if acc.dtype != torch.int64 or not acc.is_cuda or acc.numel() < 2 or not acc.is_contiguous():
            raise ValueError("acc must be a contiguous CUDA int64 tensor of at least 2 elements")
        check(self._lib.msplat_cuda_frame_pair_counts_device(self.handle, ptr(acc)))

    def enable_stage_timing(self, on: bool = True) -> None:
        check(self._lib.msplat_cuda_ctx_set_option(self.handle, b"stage_timing", int(on)))

    def drain_stage_times(self):
        """{stage: (total ms, calls)} accumulated since the last drain."""
        ms = (C.c_double * 8)()
        calls = (C.c_int64 * 8)()
        names = (C.c_char_p * 8)()
        n = C.c_int()
        check(self._lib.msplat_cuda_drain_stage_times(self.handle, C.cast(ms, C.c_void_p), C.cast(calls, C.c_void_p),
                                                      8, C.byref(n), C.cast(names, C.c_void_p)))
        return {names[i].decode(): (float(ms[i]), int(calls[i])) for i in range(n.value)}

    def sync(self) -> None:
        check(self._lib.msplat_cuda_sync(self.handle))

    def cleanup(self) -> None:
        check(self._lib.msplat_cuda_cleanup(self.handle))
