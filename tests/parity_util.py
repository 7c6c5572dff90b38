"""Comparison helpers for parity tests. Tolerances (from the path's contract):
images max-abs <= 1e-5, gradients relative L2 <= 1e-4, integer data bit-exact."""
import numpy as np

IMAGE_ATOL = 1e-5
GRAD_RTOL_L2 = 1e-4


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return float(d / n) if n > 0 else float(d)


def max_abs(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b))) if a.size else 0.0


def splat_fields(splats: np.ndarray):
    """Split the CUDA frame's splat records (N x 12) into xys, conics, colors, depths."""
    s = np.asarray(splats, np.float32).reshape(-1, 12)
    return {"xys": s[:, 0:2], "conics": s[:, 2:5], "opacity": s[:, 5], "colors": s[:, 6:9], "depths": s[:, 9]}


BACKGROUND = np.array([0.6130, 0.0101, 0.3984], np.float32)  # Model's default (core/src/model.cpp:76)
C1_LRS = [1.6e-4, 5e-3, 1e-3, 2.5e-3, 2.5e-3, 0.05]   # means, scales, quats, SH dc, SH rest, opacity
