"""Prior-guided training for street captures: the host side around PriorStep.

Restates the reference's prior plumbing (everything off by default):
 * PriorOptions (core/include/model.hpp:15-33);
 * per-camera prior maps at their own resolution -- depth (scene units, 0 = invalid),
   confidence, sky mask and keep mask packed into the (h, w, 4) byte map the kernels
   read (Camera::loadPriors, core/src/priors.cpp:202-265), with the nearest-neighbour
   resampling and the 1024-pixel cap it applies (:152-163, core/include/priors.hpp:33);
 * the priors/ directory layout, keyed by image name (attachPriors, priors.cpp:167-197);
 * the log-linear depth-weight schedule (Model::depthWeightAt, core/src/model.cpp:693-701);
 * the sky's equirect frame from the training cameras and its initial texture from
   their sky-mask pixels (computeSkyFrame / initSkyTexture, model.cpp:703-809);
 * the per-step PriorStep of a training camera and of a render (trainPriorStep /
   renderPriorStep, model.cpp:548-625).
Files are read with numpy (.npy) and Pillow (.png / .jpg masks).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .camera import expf, logf

MAX_PRIOR_DIM = 1024  # core/include/priors.hpp:33


@dataclass
class PriorOptions:
    """core/include/model.hpp:15-33 (PriorOptions), same defaults."""
    depth_weight: float = 0.0         # log-depth prior loss weight at the first step (0 = off)
    depth_weight_final: float = -1.0  # weight at the last step, log-linear in between (< 0: constant)
    depth_huber_delta: float = 0.05
    depth_min_alpha: float = 0.25
    sky_alpha_weight: float = 0.0     # push alpha to 0 on sky-mask pixels
    fill_weight: float = 0.0          # push alpha to 1 on non-sky pixels
    use_masks: bool = False           # drop gradients where the keep mask is 0
    learn_sky: bool = False
    sky_width: int = 512
    sky_height: int = 128
    sky_lr: float = 0.01
    exposure: bool = False
    exposure_lr: float = 5e-3
    exposure_reg: float = 1e-2
    max_scale_ratio: float = 0.0      # cap largest / median scale (<= 1: off)

    def active(self) -> bool:
        """Model::priorsActive (model.cpp:685-691)."""
        return (self.depth_weight > 0 or self.sky_alpha_weight > 0 or self.fill_weight > 0 or self.use_masks
                or self.learn_sky or self.exposure or self.max_scale_ratio > 1.0)

    def wants_prior_files(self) -> bool:
        return (self.depth_weight > 0 or self.sky_alpha_weight > 0 or self.fill_weight > 0 or self.use_masks
                or self.learn_sky)


@dataclass
class CameraPrior:
    """One camera's prior maps as the kernels read them."""
    depth: np.ndarray   # (h, w) float32, scene units, 0 = invalid
    aux: np.ndarray     # (h, w, 4) uint8: confidence * 255, sky 255/0, keep 255/0, 0
    has_depth: bool
    has_sky: bool
    has_mask: bool

    @property
    def width(self) -> int:
        return int(self.depth.shape[1])

    @property
    def height(self) -> int:
        return int(self.depth.shape[0])


def resample_nearest(src: np.ndarray, dw: int, dh: int) -> np.ndarray:
    """Nearest-neighbour resample of an (h, w) map, sampling pixel centres
    (resampleNearest, priors.cpp:152-163)."""
    sh, sw = src.shape[:2]
    if (sw, sh) == (dw, dh):
        return src
    ys = np.minimum(sh - 1, ((np.arange(dh, dtype=np.float32) + np.float32(0.5)) * np.float32(sh)
                             / np.float32(dh)).astype(np.int64))
    xs = np.minimum(sw - 1, ((np.arange(dw, dtype=np.float32) + np.float32(0.5)) * np.float32(sw)
                             / np.float32(dw)).astype(np.int64))
    return src[ys[:, None], xs[None, :]]


def _fit(sw: int, sh: int):
    """Size capped at MAX_PRIOR_DIM a side: lround(side * s) in float, as the reference."""
    s = min(np.float32(1.0), np.float32(MAX_PRIOR_DIM) / np.float32(max(sw, sh)))
    lround = lambda v: int(math.floor(float(np.float32(v) * s) + 0.5))  # noqa: E731 (positive values)
    return max(1, lround(sw)), max(1, lround(sh))


def _plane(a, name: str) -> np.ndarray:
    a = np.asarray(a)
    if a.ndim == 3 and a.shape[2] == 1:
        a = a[:, :, 0]
    if a.ndim != 2:
        raise ValueError(f"prior {name} must be a 2-D (H, W) array, got shape {a.shape}")
    return a.astype(np.float32)


def build_camera_prior(depth=None, confidence=None, sky=None, mask=None, depth_scale: float = 1.0,
                       use_mask: bool = False) -> Optional[CameraPrior]:
    """Camera::loadPriors (priors.cpp:202-265) over in-memory maps: depth (H, W) in
    dataset units, confidence (H, W) in [0, 1], sky / mask as (H, W) or (H, W, 3)
    images in [0, 1] (RGB averaged; a pixel is sky / kept above 0.5). The maps are
    fitted to at most 1024 pixels a side (the depth's size, else the first mask's) by
    nearest-neighbour resampling."""
    if depth is None and sky is None and not (use_mask and mask is not None):
        return None
    w = h = 0
    d = c = s = k = None
    if depth is not None:
        d0 = _plane(depth, "depth")
        w, h = _fit(d0.shape[1], d0.shape[0])
        d = resample_nearest(d0, w, h)
        if confidence is not None:
            c = resample_nearest(_plane(confidence, "confidence"), w, h)

    def grey(m, name):
        nonlocal w, h
        g = np.asarray(m, np.float32)
        if g.ndim == 3:
            g = (g[..., 0] + g[..., 1] + g[..., 2]) * np.float32(1.0 / 3.0)
        g = _plane(g, name)
        if w == 0:
            w, h = _fit(g.shape[1], g.shape[0])
        return resample_nearest(g, w, h)

    if sky is not None:
        s = grey(sky, "sky")
    if mask is not None and use_mask:
        k = grey(mask, "mask")
    n = w * h
    dd = np.zeros(n, np.float32) if d is None else d.reshape(-1).astype(np.float32).copy()
    dd[~np.isfinite(dd) | (dd <= 0)] = 0.0
    cc = np.zeros(n, np.float32)
    valid = dd > 0
    if valid.any():
        cv = np.ones(n, np.float32) if c is None else c.reshape(-1).astype(np.float32)
        cv = np.where(np.isfinite(cv), np.clip(cv, 0.0, 1.0), 0.0).astype(np.float32)
        cc[valid] = cv[valid]
    aux = np.zeros((n, 4), np.uint8)
    # lround(c * 255) of a non-negative float product
    aux[:, 0] = np.floor((cc * np.float32(255.0)).astype(np.float64) + 0.5).astype(np.uint8)
    aux[:, 1] = 0 if s is None else np.where(s.reshape(-1) > 0.5, 255, 0)
    aux[:, 2] = 255 if k is None else np.where(k.reshape(-1) > 0.5, 255, 0)
    return CameraPrior((dd * np.float32(depth_scale)).reshape(h, w).astype(np.float32), aux.reshape(h, w, 4),
                       d is not None, s is not None, k is not None)


def prior_paths(image_name: str, prior_dir: str):
    """Files of one camera under a priors/ directory (attachPriors, priors.cpp:167-197):
    depth/<name>.npy, confidence/<name>.npy, sky/<name>.png|.jpg, mask/<name>.png|.jpg,
    <name> = the image path relative to the image root without its extension, falling
    back to the bare file stem."""
    rel = os.path.splitext(image_name)[0]
    keys = [rel]
    if os.path.dirname(rel):
        keys.append(os.path.basename(rel))

    def find(sub, exts):
        for k in keys:
            for e in exts:
                p = os.path.join(prior_dir, sub, k + e)
                if os.path.exists(p):
                    return p
        return None

    return {"depth": find("depth", [".npy"]), "confidence": find("confidence", [".npy"]),
            "sky": find("sky", [".png", ".jpg"]), "mask": find("mask", [".png", ".jpg"])}


def load_camera_prior(paths: dict, depth_scale: float = 1.0, use_mask: bool = False) -> Optional[CameraPrior]:
    """Reads a camera's prior files (prior_paths) and packs them (build_camera_prior)."""
    def img(p):
        if p is None:
            return None
        from PIL import Image
        return np.asarray(Image.open(p).convert("RGB"), np.float32) / np.float32(255.0)

    depth = np.load(paths["depth"]) if paths.get("depth") else None
    conf = np.load(paths["confidence"]) if paths.get("confidence") and depth is not None else None
    return build_camera_prior(depth, conf, img(paths.get("sky")), img(paths.get("mask")) if use_mask else None,
                              depth_scale, use_mask)


def depth_weight_at(opts: PriorOptions, step: int, max_steps: int) -> float:
    """Model::depthWeightAt (model.cpp:693-701), in float32 like the reference."""
    f = np.float32
    w0, w1 = f(opts.depth_weight), f(opts.depth_weight_final)
    if w0 <= 0:
        return 0.0
    if w1 < 0:
        return float(w0)
    t = f(min(max(f(step) / f(max(1, max_steps)), f(0)), f(1)))
    if w1 == 0:
        return float(w0 * (f(1) - t))
    return float(expf(logf(w0) * (f(1) - t) + logf(w1) * t))


def compute_sky_frame(cam_to_worlds: Sequence[np.ndarray]) -> np.ndarray:
    """Equirect frame of the sky: zenith = mean camera up, azimuth 0 = mean heading,
    (up, e1, e2) as 9 floats (computeSkyFrame, model.cpp:703-738; OpenGL poses, whose
    columns are camera X, Y (up), Z (back))."""
    up = [0.0, 0.0, 0.0]
    fwd = [0.0, 0.0, 0.0]
    for m in cam_to_worlds:
        m = np.asarray(m, np.float32)
        for k in range(3):
            up[k] += float(m[k, 1])
            fwd[k] -= float(m[k, 2])

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    def norm(v):
        n = math.sqrt(dot(v, v))
        if n < 1e-12:
            return None
        return [v[0] / n, v[1] / n, v[2] / n]

    u = norm(up)
    up = [0.0, 1.0, 0.0] if u is None else u
    d = dot(fwd, up)
    f2 = norm([fwd[k] - d * up[k] for k in range(3)])
    if f2 is None:  # heading parallel to up: the world axis least aligned with up
        a = 0
        for k in (1, 2):
            if abs(up[k]) < abs(up[a]):
                a = k
        e = [0.0, 0.0, 0.0]
        e[a] = 1.0
        d = dot(e, up)
        f2 = norm([e[k] - d * up[k] for k in range(3)])
    fwd = f2
    e2 = [up[1] * fwd[2] - up[2] * fwd[1], up[2] * fwd[0] - up[0] * fwd[2], up[0] * fwd[1] - up[1] * fwd[0]]
    return np.array(up + fwd + e2, np.float32)


def init_sky_texture(views, cam_priors: List[Optional[CameraPrior]], frame: np.ndarray, W: int, H: int) -> np.ndarray:
    """Initial sky texture (initSkyTexture, model.cpp:743-809): the sky-mask pixels of
    the training images (every stride-th, stride = max(1, max(w, h) // 256)) splatted
    to the texel their ray hits; texels no image saw take their elevation row's mean,
    or the nearest row's that has data, or the mean of all sky samples (an overcast
    default when none was seen). ``views`` carry cam_to_world, fx, fy, cx, cy, image."""
    f = np.float32
    sums = np.zeros((H * W, 3), np.float64)
    cnt = np.zeros(H * W, np.float64)
    fr = np.asarray(frame, np.float32)
    for v, cp in zip(views, cam_priors):
        if cp is None or not cp.has_sky or v.image is None:
            continue
        img = np.asarray(v.image, np.float32)
        ih, iw = img.shape[:2]
        stride = max(1, max(iw, ih) // 256)
        ys = np.arange(0, ih, stride)
        xs = np.arange(0, iw, stride)
        qy = np.minimum(cp.height - 1, ((ys.astype(np.float32) + f(0.5)) * f(cp.height) / f(ih)).astype(np.int64))
        qx = np.minimum(cp.width - 1, ((xs.astype(np.float32) + f(0.5)) * f(cp.width) / f(iw)).astype(np.int64))
        yy, xx = np.meshgrid(ys, xs, indexing="ij")
        sky = cp.aux[qy[:, None], qx[None, :], 1] >= 128
        yy, xx = yy[sky], xx[sky]
        if yy.size == 0:
            continue
        M = np.asarray(v.cam_to_world, np.float32)
        dc0 = (xx.astype(np.float32) + f(0.5) - f(v.cx)) / f(v.fx)
        dc1 = (yy.astype(np.float32) + f(0.5) - f(v.cy)) / f(v.fy)
        d = [M[k, 0] * dc0 - M[k, 1] * dc1 - M[k, 2] * f(1.0) for k in range(3)]
        n = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        su = (d[0] * fr[0] + d[1] * fr[1] + d[2] * fr[2]) / n
        s1 = d[0] * fr[3] + d[1] * fr[4] + d[2] * fr[5]
        s2 = d[0] * fr[6] + d[1] * fr[7] + d[2] * fr[8]
        el = np.arcsin(np.clip(su, f(-1), f(1)))
        az = np.arctan2(s2, s1)
        u = np.floor((az / (f(2.0) * f(math.pi)) + f(0.5)) * f(W)).astype(np.int64)
        vv = np.floor((f(0.5) - el / f(math.pi)) * f(H)).astype(np.int64)
        u = ((u % W) + W) % W
        vv = np.clip(vv, 0, H - 1)
        t = vv * W + u
        c = img[yy, xx].astype(np.float64)
        np.add.at(sums, t, c)
        np.add.at(cnt, t, 1.0)
    total_n = cnt.sum()
    mean = (sums.sum(0) / total_n).astype(np.float32) if total_n > 0 else np.array([0.6, 0.7, 0.85], np.float32)
    sums = sums.reshape(H, W, 3)
    cnt = cnt.reshape(H, W)
    row_n = cnt.sum(1)
    row_has = row_n > 0
    row_mean = np.zeros((H, 3), np.float32)
    row_mean[row_has] = (sums.sum(1)[row_has] / row_n[row_has, None]).astype(np.float32)
    tex = np.zeros((H, W, 3), np.float32)
    for r in range(H):
        fill = mean
        for dv in range(H):
            if r - dv >= 0 and row_has[r - dv]:
                fill = row_mean[r - dv]
                break
            if r + dv < H and row_has[r + dv]:
                fill = row_mean[r + dv]
                break
        seen = cnt[r] > 0
        tex[r] = fill
        tex[r, seen] = (sums[r, seen] / cnt[r, seen, None]).astype(np.float32)
    return tex
