"""Seeded synthetic scenes and cameras for the splatting workloads.

The reference publishes no dataset-free benchmark, so every workload here is drawn
from fixed distributions with numpy ``default_rng(seed)``:

* means uniform in a box (``[-1,1]^3`` for the small scene, 20 x 4 x 20 m for streets),
* log-scales N(-4, 0.5) per axis,
* rotations: normalised N(0, 1) 4-vectors in (w, x, y, z) order,
* opacity logits N(0, 1),
* SH degree 3: DC N(0, 0.3), the 15 higher bases N(0, 0.05), layout (N, 15, 3).

Arrays are float32 and C-contiguous, in the layouts core/metal/bindings.h expects.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .camera import CameraSetup, look_at, prepare_cam

SH_C0 = 0.28209479177387814


@dataclass
class Gaussians:
    means: np.ndarray  # (N, 3)
    scales: np.ndarray  # (N, 3) log-scales
    quats: np.ndarray  # (N, 4) (w, x, y, z)
    features_dc: np.ndarray  # (N, 3)
    features_rest: np.ndarray  # (N, B-1, 3)
    opacities: np.ndarray  # (N, 1) logits

    @property
    def n(self) -> int:
        return int(self.means.shape[0])

    @property
    def sh_degree(self) -> int:
        b = self.features_rest.shape[1] + 1
        return 0 if b <= 1 else 1 if b <= 4 else 2 if b <= 9 else 3 if b <= 16 else 4

    def arrays(self):
        return [self.means, self.scales, self.quats, self.features_dc, self.features_rest, self.opacities]

    def copy(self) -> "Gaussians":
        return Gaussians(*[a.copy() for a in self.arrays()])


def random_gaussians(n: int, seed: int, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0), sh_degree: int = 3,
                     log_scale_mean: float = -4.0, log_scale_std: float = 0.5) -> Gaussians:
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    means = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    scales = rng.normal(log_scale_mean, log_scale_std, (n, 3)).astype(np.float32)
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opac = rng.normal(0.0, 1.0, (n, 1)).astype(np.float32)
    nb = (sh_degree + 1) ** 2
    dc = rng.normal(0.0, 0.3, (n, 3)).astype(np.float32)
    rest = rng.normal(0.0, 0.05, (n, nb - 1, 3)).astype(np.float32)
    return Gaussians(np.ascontiguousarray(means), np.ascontiguousarray(scales), q.astype(np.float32),
                     np.ascontiguousarray(dc), np.ascontiguousarray(rest), np.ascontiguousarray(opac))


# --- the small plain-method scene: 10k Gaussians, one 256x256 camera at distance 3 ---

def small_scene(seed: int = 0, n: int = 10_000) -> Gaussians:
    return random_gaussians(n, seed)


def small_camera(width: int = 256, height: int = 256, f: float = 300.0, distance: float = 3.0) -> CameraSetup:
    c2w = look_at((0.0, 0.0, distance), (0.0, 0.0, 0.0))
    return prepare_cam(c2w, width, height, f, f, width / 2.0, height / 2.0)


# --- street scale: 20 x 4 x 20 m box, cameras on a 10 m line at 1.5 m height ---

STREET_LO = (-10.0, 0.0, -10.0)
STREET_HI = (10.0, 4.0, 10.0)


def street_scene(seed: int = 0, n: int = 500_000) -> Gaussians:
    return random_gaussians(n, seed, STREET_LO, STREET_HI)


def street_camera_poses(n_views: int = 16, seed: int = 2, line_length: float = 10.0, height: float = 1.5,
                        yaw_jitter_deg: float = 30.0):
    """Camera-to-world poses evenly spaced on a line along +Z at ``height``, each looking
    along the line with a uniform yaw jitter of +-``yaw_jitter_deg``."""
    rng = np.random.default_rng(seed)
    poses = []
    for i in range(n_views):
        z = -line_length / 2 + line_length * (i / max(n_views - 1, 1))
        yaw = math.radians(rng.uniform(-yaw_jitter_deg, yaw_jitter_deg))
        eye = np.array([0.0, height, z])
        target = eye + np.array([math.sin(yaw), 0.0, math.cos(yaw)])
        poses.append(look_at(eye, target))
    return poses


def street_cameras(width: int = 1024, height: int = 512, f: float = 512.0, n_views: int = 16, seed: int = 2):
    return [prepare_cam(p, width, height, f, f, width / 2.0, height / 2.0)
            for p in street_camera_poses(n_views, seed)]


def jittered_init_points(gt: Gaussians, n: int, seed: int = 3, sigma: float = 0.05):
    """Training start points: ``n`` ground-truth means with N(0, sigma) jitter, plus the
    RGB of their DC colour as uint8 (the input msplat_init_gaussians takes)."""
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(gt.n, size=n, replace=False))
    pts = (gt.means[idx] + rng.normal(0.0, sigma, (n, 3))).astype(np.float32)
    rgb = np.clip(0.5 + SH_C0 * gt.features_dc[idx], 0.0, 1.0)
    return np.ascontiguousarray(pts), np.ascontiguousarray((rgb * 255.0).astype(np.uint8))


# --- serving: cameras on a sphere of radius 5 facing the centre ---

def sphere_pose(rng: np.random.Generator, radius: float = 5.0) -> np.ndarray:
    """Camera-to-world pose at a uniform point of a sphere of ``radius``, facing its centre."""
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    up = (0.0, 1.0, 0.0) if abs(v[1]) < 0.95 else (1.0, 0.0, 0.0)
    return look_at(radius * v, (0.0, 0.0, 0.0), up)


def sphere_camera(rng: np.random.Generator, width: int, height: int, radius: float = 5.0,
                  f_scale: float = 1.0) -> CameraSetup:
    """A pinhole camera (60 degree horizontal field of view) at sphere_pose."""
    pose = sphere_pose(rng, radius)
    f = f_scale * 0.5 * width / math.tan(math.radians(30.0))
    return prepare_cam(pose, width, height, f, f, width / 2.0, height / 2.0)
