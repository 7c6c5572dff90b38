"""Module-level functions of the reference's ``msplat._core`` for this backend.

Mirrors the GPU primitive hooks and utilities of python/bindings.cpp:655-778: numpy
in, numpy out, computed on the GPU through the C-ABI, with the same argument
checks and error types (ValueError where the reference raises invalid_argument).
"""
from __future__ import annotations

import numpy as np
import torch

from .backend import Context

_ctx = None


def _context() -> Context:
    global _ctx
    if _ctx is None:
        _ctx = Context()
    return _ctx


def _gpu_radix_sort(keys: np.ndarray, key_bits: int = 64):
    """Stable GPU radix sort of uint64 keys. Returns (sorted_keys, order) as the
    reference's hook does (python/bindings.cpp:656-677)."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    if keys.ndim != 1:
        raise ValueError("keys must be one-dimensional")
    n = keys.size
    if n == 0:
        return np.zeros(0, np.uint64), np.zeros(0, np.uint32)
    k = torch.from_numpy(keys.view(np.int64)).cuda()
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    ctx = _context()
    ctx.radix_sort(k, v, int(key_bits))
    torch.cuda.current_stream().synchronize()
    return k.cpu().numpy().view(np.uint64), v.cpu().numpy().view(np.uint32)


def _gpu_knn3_mean_dist(points: np.ndarray) -> np.ndarray:
    """Exact mean distance to the 3 nearest other points (python/bindings.cpp:678-690)."""
    pts = np.ascontiguousarray(points, dtype=np.float32)
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise ValueError("points must have shape (N, 3)")
    if pts.shape[0] == 0:
        raise ValueError("points must not be empty")
    out = _context().knn3_mean_dist(torch.from_numpy(pts).cuda())
    return out.cpu().numpy()


def sync() -> None:
    """Synchronize the GPU (wait for all queued work)."""
    torch.cuda.synchronize()


def cleanup() -> None:
    """Release the cached GPU buffers of the module's context."""
    global _ctx
    if _ctx is not None:
        _ctx.cleanup()
        _ctx = None
