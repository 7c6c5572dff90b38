"""Autotuner for the rasterizer's staging sizes and the batched forward's block shape.

The forward and backward rasterizers stage each tile's depth-sorted Gaussians in
shared memory in rounds; the backward also reduces its per-pixel gradients in
sub-batches through a transposed shared-memory buffer. The round sizes trade shared
memory (and so resident blocks per SM) against synchronisation and staging overhead,
and the best choice depends on the workload (Gaussians per tile, image sizes, views
per step). The library compiles a fixed set of variants (msplat_cuda_raster_variant);
every variant computes the same images and gradients, so the tuner only times them:
it runs the caller's step on each variant, interleaved over several rounds to share
out drift (training changes the scene as it goes), and keeps the fastest.

The batched forward also has a block shape (msplat_cuda_raster_shape): a block
composites a whole 16 x 16 tile, a 16 x 8 half or an 8 x 8 quarter of it, the last
being the reference Metal rasterizer's thread group inside its 16 x 16 bins
(core/metal/msplat_metal.mm:1187-1197). Every shape walks the tile's whole list, so
the tile binning itself stays the reference's BLOCK_X / BLOCK_Y (core/cpu/
msplat_cpu.cpp:27) -- which Gaussians a pixel evaluates, and so parity, depend on it
-- and the shape only moves work between blocks: smaller blocks repeat the staging of
each round and finish their pixels independently.
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


def raster_shapes() -> List[dict]:
    """The batched forward's block shapes: pixels a block composites."""
    w, h = C.c_int32(), C.c_int32()
    n = lib().msplat_cuda_raster_shape(0, C.byref(w), C.byref(h))
    out = []
    for s in range(n):
        lib().msplat_cuda_raster_shape(s, C.byref(w), C.byref(h))
        out.append({"shape": s, "w": w.value, "h": h.value})
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
                warmup: int = 2, reps: int = 6, rounds: int = 2, shapes: Optional[Sequence[int]] = None) -> Dict:
    """Time ``step`` on each rasterizer variant and batched-forward block shape (set on
    every context in ``contexts``; ``shapes`` None keeps each context's shape), keep the
    fastest pair, and return {"best": v, "best_shape": s, "ms": {v: median}} -- with
    "ms" keyed "v/s" when more than one shape is swept."""
    vs = list(variants) if variants is not None else [d["variant"] for d in raster_variants()]
    ss = list(shapes) if shapes is not None else [None]
    points = [(v, s) for s in ss for v in vs]
    samples: Dict[tuple, List[float]] = {pt: [] for pt in points}
    for _ in range(rounds):
        for v, s in points:
            for c in contexts:
                c.set_raster_variant(v)
                if s is not None:
                    c.set_raster_shape(s)
            for _ in range(warmup):
                step()
            samples[(v, s)].append(time_steps(step, reps))
    med = {pt: statistics.median(x) for pt, x in samples.items()}
    bv, bs = min(med, key=med.get)
    for c in contexts:
        c.set_raster_variant(bv)
        if bs is not None:
            c.set_raster_shape(bs)
    ms = {v: m for (v, _), m in med.items()} if len(ss) == 1 else {f"{v}/{s}": m for (v, s), m in med.items()}
    return {"best": bv, "best_shape": bs, "ms": ms,
            "variants": {d["variant"]: d for d in raster_variants() if d["variant"] in vs},
            "shapes": {d["shape"]: d for d in raster_shapes() if d["shape"] in ss}}
