"""Camera set-up for the splatting path.

Restates ``Model::prepareCam`` (core/src/model.cpp:498-546): an OpenGL camera-to-world
pose (4x4 row-major, camera looking down -Z with +Y up) becomes the world-to-camera
``viewmat`` with the Y/Z axes negated (model.cpp:514-521), the full projection
``projmat = P(n=0.001, f=1000) @ viewmat`` (model.cpp:522-525), the camera position,
and the 16x16 tile grid (model.cpp:538-540). All arithmetic is float32, as in the
reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TILE = 16


@dataclass
class CameraSetup:
    """Everything ``msplat_render`` / ``msplat_train_step`` take about one view."""

    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    viewmat: np.ndarray  # (4, 4) float32, row-major world-to-camera
    projmat: np.ndarray  # (4, 4) float32, row-major clip-from-world
    cam_pos: np.ndarray  # (3,) float32
    tiles_x: int = field(init=False)
    tiles_y: int = field(init=False)

    def __post_init__(self):
        self.tiles_x = (self.width + TILE - 1) // TILE
        self.tiles_y = (self.height + TILE - 1) // TILE

    @property
    def tile_bounds(self):
        return (self.tiles_x, self.tiles_y, 1)


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """OpenGL camera-to-world pose at ``eye`` looking at ``target`` (row-major 4x4)."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    true_up = np.cross(right, fwd)
    c2w = np.eye(4)
    c2w[:3, 0] = right
    c2w[:3, 1] = true_up
    c2w[:3, 2] = -fwd  # OpenGL: the camera looks along -Z
    c2w[:3, 3] = eye
    return c2w.astype(np.float32)


def prepare_cam(cam_to_world, width: int, height: int, fx: float, fy: float, cx: float, cy: float) -> CameraSetup:
    """Model::prepareCam (core/src/model.cpp:498-546) for one full-resolution view."""
    d = np.asarray(cam_to_world, np.float32).reshape(4, 4)
    f32 = np.float32
    R = np.empty((3, 3), np.float32)
    T = np.empty(3, np.float32)
    for i in range(3):
        R[i, 0] = d[i, 0]
        R[i, 1] = -d[i, 1]
        R[i, 2] = -d[i, 2]
        T[i] = d[i, 3]
    Rinv = R.T.copy()
    Tinv = np.empty(3, np.float32)
    for i in range(3):
        Tinv[i] = -(f32(Rinv[i, 0] * T[0]) + f32(Rinv[i, 1] * T[1]) + f32(Rinv[i, 2] * T[2]))
    vm = np.array(
        [[Rinv[0, 0], Rinv[0, 1], Rinv[0, 2], Tinv[0]],
         [Rinv[1, 0], Rinv[1, 1], Rinv[1, 2], Tinv[1]],
         [Rinv[2, 0], Rinv[2, 1], Rinv[2, 2], Tinv[2]],
         [0, 0, 0, 1]], np.float32)
    fov_x = f32(2.0) * f32(math.atan(f32(width) / (f32(2.0) * f32(fx))))
    fov_y = f32(2.0) * f32(math.atan(f32(height) / (f32(2.0) * f32(fy))))
    t_p = f32(0.001) * f32(math.tan(f32(0.5) * fov_y))
    r_p = f32(0.001) * f32(math.tan(f32(0.5) * fov_x))
    pm = np.array(
        [[f32(0.001) / r_p, 0, 0, 0],
         [0, f32(0.001) / t_p, 0, 0],
         [0, 0, f32(1000.001) / f32(999.999), f32(-1000.0 * 0.001) / f32(999.999)],
         [0, 0, 1, 0]], np.float32)
    pvm = np.zeros((4, 4), np.float32)
    for i in range(4):
        for j in range(4):
            acc = f32(0.0)
            for k in range(4):
                acc = f32(acc + f32(pm[i, k] * vm[k, j]))
            pvm[i, j] = acc
    return CameraSetup(int(width), int(height), float(fx), float(fy), float(cx), float(cy), vm, pvm,
                       T.astype(np.float32).copy())
