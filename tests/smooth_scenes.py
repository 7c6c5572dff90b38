"""Smooth scenes for finite-difference gradient checks (test infrastructure).

As in the reference's tests/gradcheck.cpp:5-9, the Gaussians are wider than the
image and faint enough that no cut-off (sigma 5.55, alpha 1/255, alpha 0.999,
transmittance 1e-4, tile rectangle) moves while a parameter is perturbed by h, so
finite differences see the same function the backward differentiates. The camera is
rotated and translated and the quaternions are not unit length.
"""
import math

import numpy as np

from msplat_street_b200.camera import prepare_cam
from msplat_street_b200.scenes import Gaussians


def _rot(a, b, c):
    Rz = np.array([[math.cos(c), -math.sin(c), 0], [math.sin(c), math.cos(c), 0], [0, 0, 1]])
    Ry = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    Rx = np.array([[1, 0, 0], [0, math.cos(b), -math.sin(b)], [0, math.sin(b), math.cos(b)]])
    return Rz @ Ry @ Rx


def smooth_scene(n=64, width=32, height=32, seed=1234, view_dependent=False, sh_degree=3):
    rng = np.random.default_rng(seed)
    fx, fy = 40.0, 38.0
    R = _rot(0.2, -0.15, 0.1)                 # camera from world rotation
    t = np.array([0.3, -0.2, 0.5])
    c2w = np.eye(4)
    # prepare_cam negates Y/Z of the camera-to-world rotation (OpenGL -> OpenCV)
    c2w[:3, :3] = R.T @ np.diag([1.0, -1.0, -1.0])
    c2w[:3, 3] = -R.T @ t
    cam = prepare_cam(c2w.astype(np.float32), width, height, fx, fy, width / 2 + 0.4, height / 2 - 0.3)
    Rc = cam.viewmat[:3, :3].astype(np.float64)
    tc = cam.viewmat[:3, 3].astype(np.float64)
    means = np.zeros((n, 3))
    scales = np.zeros((n, 3))
    for i in range(n):
        z = 2.5 + 0.03 * i
        pc = np.array([rng.uniform(-0.15, 0.15) * z, rng.uniform(-0.15, 0.15) * z, z])
        means[i] = Rc.T @ (pc - tc)
        scales[i] = np.log(rng.uniform(26.0, 36.0, 3) * z / fx)
    q = rng.uniform(-1, 1, (n, 4))
    q = 1.3 * q / np.linalg.norm(q, axis=1, keepdims=True)
    dc = rng.uniform(-0.6, 0.6, (n, 3))
    k = (sh_degree + 1) ** 2 - 1
    rest = rng.uniform(-0.15, 0.15, (n, k, 3)) if view_dependent else np.zeros((n, k, 3))
    opac = rng.uniform(-3.5, -1.5, (n, 1))
    g = Gaussians(*[np.ascontiguousarray(a, np.float32) for a in (means, scales, q, dc, rest, opac)])
    yy, xx = np.mgrid[0:height, 0:width]
    gt = np.stack([0.5 + 0.3 * np.sin(0.21 * xx + 0.7 * c) * np.cos(0.17 * yy - 0.3 * c) for c in range(3)], -1)
    gt = (gt + rng.uniform(-0.05, 0.05, gt.shape)).astype(np.float32)
    return g, cam, np.ascontiguousarray(gt)
