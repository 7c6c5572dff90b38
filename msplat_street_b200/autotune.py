"""Autotuner for the rasterizer's staging sizes.

The forward and backward rasterizers stage each tile's depth-sorted Gaussians in
shared memory in rounds; the backward also reduces its per-pixel gradients in
sub-batches through a transposed shared-memory buffer. The round sizes trade shared
memory (and so resident blocks per SM) against synchronisation and staging overhead,
and the best choice depends on the workload (Gaussians per tile, image sizes, views
per step). The library compiles a fixed set of variants (msplat_cuda_raster_variant);
every variant computes the same images and gradients, so the tuner only times them:
it runs the caller's step on each variant, interleaved over several rounds to share
out drift (training changes the scene as it goes), and keeps the fastest.

The reference has no counterpart (its Metal backend fixes the tile size and batch,
core/metal/msplat_metal.mm); the tile shape itself stays 16 x 16, the reference's
BLOCK_X / BLOCK_Y (core/cpu/msplat_cpu.cpp:27), which the tile keys and the parity
with the reference depend on.
"""
from __future__ import annotations

import ctypes as C
import statistics
from typing import Callable, Dict, List, Optional, Sequence

import torch

from ._lib import lib


def raster_variants() -> List[dict]:
    """The compiled variants: Gaussians staged per forward round, per backward round,
    and the backward reduction's sub-batch."""
    f, b, s = C.c_int32(), C.c_int32(), C.c_int32()
    n = lib().msplat_cuda_raster_variant(0, C.byref(f), C.byref(b), C.byref(s))
    out = []
    for v in range(n):
        lib().msplat_cuda_raster_variant(v, C.byref(f), C.byref(b), C.byref(s))
        out.append({"variant": v, "fwd_batch": f.value, "bwd_batch": b.value, "bwd_sub": s.value})
    return out


def time_steps(step: Callable[[], object], n: int) -> float:
    """Milliseconds per call of ``step`` over ``n`` calls, between device synchronisations."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(n):
        step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / n


def tune_raster(contexts: Sequence, step: Callable[[], object], variants: Optional[Sequence[int]] = None,
                warmup: int = 2, reps: int = 6, rounds: int = 2) -> Dict:
    """Time ``step`` on each rasterizer variant (set on every context in
    ``contexts``), keep the fastest set, and return {"best": v, "ms": {v: median}}."""
    vs = list(variants) if variants is not None else [d["variant"] for d in raster_variants()]
    samples: Dict[int, List[float]] = {v: [] for v in vs}
    for _ in range(rounds):
        for v in vs:
            for c in contexts:
                c.set_raster_variant(v)
            for _ in range(warmup):
                step()
            samples[v].append(time_steps(step, reps))
    ms = {v: statistics.median(x) for v, x in samples.items()}
    best = min(ms, key=ms.get)
    for c in contexts:
        c.set_raster_variant(best)
    return {"best": best, "ms": ms, "variants": {d["variant"]: d for d in raster_variants() if d["variant"] in ms}}
