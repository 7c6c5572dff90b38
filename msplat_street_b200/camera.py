"""Camera set-up for the splatting path.

Restates ``Model::prepareCam`` (core/src/model.cpp:498-546): an OpenGL camera-to-world
pose (4x4 row-major, camera looking down -Z with +Y up) becomes the world-to-camera
``viewmat`` with the Y/Z axes negated (model.cpp:514-521), the full projection
``projmat = P(n=0.001, f=1000) @ viewmat`` (model.cpp:522-525), the camera position,
and the 16x16 tile grid (model.cpp:538-540), at a resolution-schedule level: the
level's whole-pixel size (``levelSize``, core/include/image_sizing.hpp:62) and the
intrinsics scaled by the actual per-axis ratio (model.cpp:500-508). All arithmetic is
float32 in the reference's order, and the reference's float ``std::atan`` /
``std::tan`` are the C library's ``atanf`` / ``tanf``, called here through ctypes, so
the matrices are the reference's bit for bit.
"""
from __future__ import annotations

import ctypes
import ctypes.util
from dataclasses import dataclass, field

import numpy as np

TILE = 16


def _libm():
    lib = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    for name in ("atanf", "tanf", "logf", "expf"):
        fn = getattr(lib, name)
        fn.restype = ctypes.c_float
        fn.argtypes = [ctypes.c_float]
    lib.powf.restype = ctypes.c_float
    lib.powf.argtypes = [ctypes.c_float, ctypes.c_float]
    return lib


LIBM = _libm()


def atanf(x) -> np.float32:
    return np.float32(LIBM.atanf(float(x)))


def tanf(x) -> np.float32:
    return np.float32(LIBM.tanf(float(x)))


def logf(x) -> np.float32:
    return np.float32(LIBM.logf(float(x)))


def expf(x) -> np.float32:
    return np.float32(LIBM.expf(float(x)))


def powf(x, y) -> np.float32:
    return np.float32(LIBM.powf(float(x), float(y)))


def level_size(full: int, factor: int) -> int:
    """levelSize (core/include/image_sizing.hpp:62): a schedule level's pixel size."""
    return int(full) if factor <= 1 else int(full) // int(factor)


def schedule_downscale_factor(step: int, num_downscales: int, resolution_schedule: int) -> int:
    """scheduleDownscaleFactor (core/src/image_sizing.cpp:129-133): 2^(downscales left)."""
    if num_downscales <= 0 or resolution_schedule <= 0:
        return 1
    remaining = num_downscales - int(step) // int(resolution_schedule)
    return 1 << min(max(remaining, 0), 30)


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


def prepare_cam(cam_to_world, width: int, height: int, fx: float, fy: float, cx: float, cy: float,
                factor: int = 1) -> CameraSetup:
    """Model::prepareCam (core/src/model.cpp:498-546) for one view at downscale
    ``factor`` (1 = full resolution)."""
    d = np.asarray(cam_to_world, np.float32).reshape(4, 4)
    f32 = np.float32
    w, h = level_size(width, factor), level_size(height, factor)
    rx = f32(w) / f32(width) if width > 0 else f32(1.0) / f32(factor)
    ry = f32(h) / f32(height) if height > 0 else f32(1.0) / f32(factor)
    fx, cx = f32(fx) * rx, f32(cx) * rx
    fy, cy = f32(fy) * ry, f32(cy) * ry
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
    fov_x = f32(2.0) * atanf(f32(w) / (f32(2.0) * fx))
    fov_y = f32(2.0) * atanf(f32(h) / (f32(2.0) * fy))
    t_p = f32(0.001) * tanf(f32(0.5) * fov_y)
    r_p = f32(0.001) * tanf(f32(0.5) * fov_x)
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
    return CameraSetup(int(w), int(h), float(fx), float(fy), float(cx), float(cy), vm, pvm,
                       T.astype(np.float32).copy())
