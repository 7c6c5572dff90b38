"""Render serving: many trained scenes resident in HBM, continuous batching of camera
requests into the persistent multi-view rasterizer.

The reference renders one view per call (msplat_render, core/metal/bindings.h:81-91,
driven by Model::render / render_from_pose, core/src/model.cpp:548-583); it has no
server. This module is the serving form built on the batched entry point
(msplat_cuda_render_batch):

* ``SceneStore`` keeps scenes' parameter arrays on the device under a byte budget.
  A scene is admitted (uploaded from its pinned host copy) when a request needs it;
  when the budget is full the least recently used scene that no batch in flight
  holds is evicted. A scene larger than the whole budget is rejected at ``add``.
* ``RenderServer`` runs ``slots`` workers, each with its own context and CUDA stream.
  A free worker takes every request that has arrived (up to ``max_batch`` requests
  and ``max_batch_pixels`` pixels, first come first served) whose scene can be made
  resident, renders them with one batched call and delivers the images. Requests
  that arrive while other batches are on the GPU are taken by the next free worker,
  so batches overlap on the device (continuous batching, not a queue in front of one
  renderer).
* ``mode="plain"`` is the baseline: one worker, one request at a time through the
  single-view msplat_cuda_render.

Every image is rendered by per-tile work that depends only on its own view (no
cross-request accumulation), so a request's image is the same, bit for bit, alone
and in any batch.
"""
from __future__ import annotations

import contextlib
import math
import threading
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from .backend import BatchItem, Context, GaussianParams
from .camera import CameraSetup
from .scenes import sphere_camera

SERVING_RESOLUTIONS = ((512, 512), (1280, 720), (1920, 1080))


def params_bytes(p: GaussianParams) -> int:
    return sum(t.numel() * t.element_size() for t in p.tensors())


def random_scene_tensors(n: int, seed: int, device="cuda", sh_degree: int = 3) -> GaussianParams:
    """A scene drawn from the serving distributions (means U[-1,1]^3, log-scales
    N(-4, 0.5), normalised N(0,1) quaternions, opacity logits N(0,1), DC N(0, 0.3),
    higher SH N(0, 0.05)), generated on ``device`` with a seeded torch generator."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    f = dict(device=device, dtype=torch.float32, generator=g)
    nb = (sh_degree + 1) ** 2
    means = torch.rand((n, 3), **f) * 2.0 - 1.0
    scales = torch.randn((n, 3), **f) * 0.5 - 4.0
    q = torch.randn((n, 4), **f)
    q = q / q.norm(dim=1, keepdim=True)
    dc = torch.randn((n, 3), **f) * 0.3
    rest = torch.randn((n, nb - 1, 3), **f) * 0.05
    opac = torch.randn((n, 1), **f)
    return GaussianParams(means.contiguous(), scales.contiguous(), q.contiguous(), dc.contiguous(),
                          rest.contiguous(), opac.contiguous())


def scene_sizes(n_scenes: int = 32, lo: int = 50_000, hi: int = 3_000_000, seed: int = 5) -> List[int]:
    """Gaussian counts log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return [int(round(math.exp(x))) for x in rng.uniform(math.log(lo), math.log(hi), n_scenes)]


@dataclass
class RenderRequest:
    scene_id: int
    camera: CameraSetup
    arrival: float = 0.0  # seconds from the start of the run
    rid: int = 0


@dataclass
class RenderResult:
    rid: int
    scene_id: int
    width: int
    height: int
    arrival: float
    start: float  # when its batch was launched
    done: float  # when its image was complete on the device
    batch_size: int
    image: Optional[torch.Tensor] = None

    @property
    def latency_ms(self) -> float:
        return (self.done - self.arrival) * 1e3


def poisson_requests(rate: float, duration: float, n_scenes: int, seed: int = 11,
                     resolutions: Sequence = SERVING_RESOLUTIONS, radius: float = 5.0) -> List[RenderRequest]:
    """Seeded Poisson arrivals at ``rate`` requests/s over ``duration`` seconds; each
    request has a uniform scene id, a uniform resolution and a pinhole camera on a
    sphere of ``radius`` around the origin, facing it."""
    rng = np.random.default_rng(seed)
    out: List[RenderRequest] = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        sid = int(rng.integers(n_scenes))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        out.append(RenderRequest(sid, sphere_camera(rng, w, h, radius=radius), t, len(out)))
    return out


class SceneStore:
    """Scenes resident on the device under a byte budget, evicted least recently used.

    ``reserved`` (a callable) reports device bytes held outside the scenes (the render
    contexts' caches and output arenas); admission keeps scenes + reserved within the
    budget."""

    def __init__(self, budget_bytes: int, device="cuda", reserved: Optional[Callable[[], int]] = None):
        self.budget = int(budget_bytes)
        d = torch.device(device)
        if d.type == "cuda" and d.index is None:
            d = torch.device("cuda", torch.cuda.current_device())
        self.device = d
        self.reserved = reserved or (lambda: 0)
        self._host: Dict[int, GaussianParams] = {}
        self._dev: "OrderedDict[int, GaussianParams]" = OrderedDict()  # least recent first
        self._ready: Dict[int, Optional[torch.cuda.Event]] = {}
        self._pins: Dict[int, int] = {}
        self._lock = threading.Lock()
        self.uploads = 0
        self.evictions = 0

    def __len__(self) -> int:
        return len(self._host)

    @property
    def resident_bytes(self) -> int:
        return sum(params_bytes(p) for p in self._dev.values())

    def resident_ids(self) -> List[int]:
        with self._lock:
            return list(self._dev.keys())

    def add(self, scene_id: int, params: GaussianParams, resident: bool = False, host_copy: bool = True) -> None:
        """Register a scene. Its host copy is kept (pinned when CUDA is present) for
        re-admission after eviction. ``resident=True`` also keeps ``params`` as the
        device copy when they already live on the store's device (no upload); a
        resident scene added with ``host_copy=False`` is never evicted."""
        nbytes = params_bytes(params)
        if nbytes > self.budget:
            raise MemoryError(f"scene {scene_id} needs {nbytes} bytes, more than the whole budget ({self.budget})")
        if not host_copy and not resident:
            raise ValueError("a scene without a host copy must be added resident")
        host = None
        if host_copy:
            host = GaussianParams(*[t.detach().to("cpu").contiguous() for t in params.tensors()])
            if torch.cuda.is_available():
                host = GaussianParams(*[t.pin_memory() for t in host.tensors()])
        with self._lock:
            if resident:
                if params.means.device != self.device:
                    raise ValueError("resident=True needs parameters on the store's device")
                if not self._make_room(nbytes):
                    raise MemoryError(f"no room for scene {scene_id}: the budget is held by scenes in use")
                self._dev[scene_id] = params
                self._ready[scene_id] = None
            self._host[scene_id] = host
            self._pins.setdefault(scene_id, 0)

    def set_budget(self, budget_bytes: int) -> None:
        """Change the budget, evicting least recently used scenes not in use until the
        residents fit (those in use stay until released)."""
        with self._lock:
            self.budget = int(budget_bytes)
            self._make_room(0)

    def _make_room(self, nbytes: int) -> bool:
        # caller holds the lock
        while self.resident_bytes + self.reserved() + nbytes > self.budget:
            victim = next((s for s in self._dev if self._pins.get(s, 0) == 0 and self._host.get(s) is not None),
                          None)
            if victim is None:
                return False
            del self._dev[victim]
            self._ready.pop(victim, None)
            self.evictions += 1
        return True

    def try_acquire(self, scene_id: int, stream: Optional[torch.cuda.Stream] = None) -> Optional[GaussianParams]:
        """The scene's device arrays, pinned until ``release``; uploads it (on
        ``stream``) when it is not resident. None when it cannot be admitted now: the
        budget is held by scenes that batches in flight are using."""
        with self._lock:
            if scene_id not in self._host:
                raise KeyError(f"unknown scene {scene_id}")
            p = self._dev.get(scene_id)
            if p is None:
                host = self._host[scene_id]
                if not self._make_room(params_bytes(host)):
                    return None
                ev = None
                if self.device.type == "cuda":
                    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
                        p = GaussianParams(*[t.to(self.device, non_blocking=True) for t in host.tensors()])
                        ev = torch.cuda.Event()
                        ev.record()
                else:
                    p = GaussianParams(*[t.clone() for t in host.tensors()])
                self._dev[scene_id] = p
                self._ready[scene_id] = ev
                self.uploads += 1
            else:
                self._dev.move_to_end(scene_id)
            self._pins[scene_id] += 1
            ev = self._ready.get(scene_id)
        if ev is not None and stream is not None:
            stream.wait_event(ev)  # an upload issued on another stream must land first
        return p

    def release(self, scene_id: int) -> None:
        with self._lock:
            if self._pins.get(scene_id, 0) <= 0:
                raise RuntimeError(f"scene {scene_id} released more often than acquired")
            self._pins[scene_id] -= 1


@dataclass
class _Worker:
    ctx: object  # a Context, or any object with render / render_batch / device_bytes
    stream: Optional[torch.cuda.Stream]
    arena: Optional[torch.Tensor] = None
    held_bytes: int = 0  # context caches + arena, refreshed by the worker's own thread
    busy_s: float = 0.0
    batches: int = 0


class RenderServer:
    """Continuous-batching render server over a ``SceneStore`` (see module doc)."""

    def __init__(self, store: SceneStore, background, slots: int = 2, max_batch: int = 32,
                 max_batch_pixels: int = 24 * 1920 * 1080, mode: str = "batched", keep_images: bool = False,
                 on_result: Optional[Callable[[RenderResult, torch.Tensor], None]] = None,
                 renderer_factory: Callable[[], object] = Context, raster_shape: Optional[int] = 1):
        if mode not in ("batched", "plain"):
            raise ValueError("mode must be 'batched' or 'plain'")
        if mode == "plain":
            slots, max_batch = 1, 1
        self.store = store
        self.background = np.ascontiguousarray(np.asarray(background, np.float32))
        self.mode = mode
        self.max_batch = int(max_batch)
        self.max_batch_pixels = int(max_batch_pixels)
        self.keep_images = keep_images
        self.on_result = on_result
        cuda = store.device.type == "cuda"
        self.workers = [_Worker(renderer_factory(), torch.cuda.Stream(store.device) if cuda else None)
                        for _ in range(int(slots))]
        # the batched forward's block shape (results do not depend on it): 16 x 8 pixel
        # blocks composite a 3 M-Gaussian 1080p frame in 0.54 ms against 0.60 ms for
        # whole 16 x 16 tiles and 0.61 ms for 8 x 8 quarters
        for w in self.workers:
            if raster_shape is not None and hasattr(w.ctx, "set_raster_shape"):
                w.ctx.set_raster_shape(raster_shape)
        self._busy = 0
        store.reserved = self.reserved_bytes

    def reserved_bytes(self) -> int:
        return sum(w.held_bytes for w in self.workers)

    def close(self) -> None:
        for w in self.workers:
            if hasattr(w.ctx, "close"):
                w.ctx.close()

    def _on_stream(self, w: _Worker):
        return torch.cuda.stream(w.stream) if w.stream is not None else contextlib.nullcontext()

    # -- batch formation -----------------------------------------------------------
    def _take(self, pending: deque, w: _Worker):
        """Pop up to max_batch arrived requests (FCFS) whose scenes can be acquired."""
        batch, params, pix = [], [], 0
        skipped = []
        while pending and len(batch) < self.max_batch:
            r = pending[0]
            npx = r.camera.width * r.camera.height
            if batch and pix + npx > self.max_batch_pixels:
                break
            pending.popleft()
            p = self.store.try_acquire(r.scene_id, w.stream)
            if p is None:
                skipped.append(r)
                continue
            batch.append(r)
            params.append(p)
            pix += npx
        for r in reversed(skipped):
            pending.appendleft(r)
        return batch, params, pix

    def _render(self, w: _Worker, batch: List[RenderRequest], params: List[GaussianParams], pix: int):
        need = pix * 3
        if w.arena is None or w.arena.numel() < need:
            with self._on_stream(w):
                w.arena = torch.empty(max(need, self.max_batch_pixels * 3 if self.mode == "batched" else need),
                                      dtype=torch.float32, device=self.store.device)
        outs, off = [], 0
        for r in batch:
            n = r.camera.width * r.camera.height * 3
            outs.append(w.arena[off:off + n].view(r.camera.height, r.camera.width, 3))
            off += n
        if self.mode == "plain":
            r, p = batch[0], params[0]
            with self._on_stream(w):
                w.ctx.render(p, r.camera, self.background, out=outs[0])
        else:
            w.ctx.render_batch([BatchItem(p, r.camera, self.background) for r, p in zip(batch, params)], outs,
                               stream=w.stream)
        return outs

    # -- the serving loop ------------------------------------------------------------
    def run(self, requests: Sequence[RenderRequest], realtime: bool = True) -> List[RenderResult]:
        """Serve ``requests`` (each released at its arrival time when ``realtime``,
        else all at once) and return one result per request, in completion order."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending: deque = deque()
        cv = threading.Condition()
        results: List[RenderResult] = []
        state = {"fed": False, "error": None}
        t0 = time.perf_counter()

        def feeder():
            for r in reqs:
                if realtime:
                    dt = t0 + r.arrival - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                with cv:
                    pending.append(r)
                    cv.notify()
            with cv:
                state["fed"] = True
                cv.notify_all()

        def worker(w: _Worker):
            try:
                while True:
                    with cv:
                        while not pending and not state["fed"] and state["error"] is None:
                            cv.wait(0.05)
                        if state["error"] is not None or (not pending and state["fed"]):
                            return
                        batch, params, pix = self._take(pending, w)
                        if not batch and self._busy == 0:
                            raise MemoryError("no request can be admitted: the budget is smaller than a scene "
                                              "plus the renderers' working memory")
                        self._busy += bool(batch)
                    if not batch:  # every arrived scene is blocked on memory: wait for a release
                        time.sleep(0.0005)
                        continue
                    start = time.perf_counter() - t0
                    try:
                        outs = self._render(w, batch, params, pix)
                        if w.stream is not None:
                            w.stream.synchronize()
                    finally:
                        for r in batch:
                            self.store.release(r.scene_id)
                        with cv:
                            self._busy -= 1
                    done = time.perf_counter() - t0
                    w.held_bytes = w.ctx.device_bytes() + (w.arena.numel() * 4 if w.arena is not None else 0)
                    w.busy_s += done - start
                    w.batches += 1
                    for r, img in zip(batch, outs):
                        res = RenderResult(r.rid, r.scene_id, r.camera.width, r.camera.height,
                                           r.arrival if realtime else 0.0, start, done, len(batch))
                        if self.keep_images:
                            res.image = img.clone()
                        if self.on_result is not None:
                            self.on_result(res, img)
                        with cv:
                            results.append(res)
                    with cv:
                        cv.notify_all()
            except BaseException as e:  # surface the first failure to the caller
                with cv:
                    if state["error"] is None:
                        state["error"] = e
                    cv.notify_all()

        threads = [threading.Thread(target=feeder, daemon=True)]
        threads += [threading.Thread(target=worker, args=(w,), daemon=True) for w in self.workers]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if state["error"] is not None:
            raise state["error"]
        if len(results) != len(reqs):
            raise RuntimeError(f"served {len(results)} of {len(reqs)} requests")
        return results


def latency_summary(results: Sequence[RenderResult], wall_s: Optional[float] = None) -> dict:
    """p50 / p99 latency (ms), frames/s, mean batch size, and the 1920x1080 p99."""
    if not results:
        return {"requests": 0}
    lat = np.array([r.latency_ms for r in results])
    first = min(r.arrival for r in results)
    last = max(r.done for r in results)
    span = wall_s if wall_s is not None else max(last - first, 1e-9)
    hd = np.array([r.latency_ms for r in results if (r.width, r.height) == (1920, 1080)])
    return {
        "requests": len(results),
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "p99_1080p_ms": float(np.percentile(hd, 99)) if hd.size else None,
        "frames_per_s": len(results) / span,
        "mean_batch": float(np.mean([r.batch_size for r in results])),
    }
