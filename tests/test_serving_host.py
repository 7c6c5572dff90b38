"""Host logic of the render server, on the CPU: scene admission against a byte budget,
LRU eviction, request streams, and continuous batching with a stand-in renderer (the
GPU path is covered by test_gpu_batch.py)."""
import threading
import time

import numpy as np
import pytest
import torch

from msplat_street_b200 import serving
from msplat_street_b200.backend import GaussianParams
from msplat_street_b200.scenes import small_camera


def _scene(n, seed=0):
    return serving.random_scene_tensors(n, seed, device="cpu", sh_degree=1)


def _nbytes(n, sh_degree=1):
    return n * (3 + 3 + 4 + 3 + ((sh_degree + 1) ** 2 - 1) * 3 + 1) * 4


def test_params_bytes_and_distributions():
    p = _scene(1000, 3)
    assert serving.params_bytes(p) == _nbytes(1000)
    assert p.sh_degree == 1
    m = p.means
    assert float(m.min()) >= -1.0 and float(m.max()) <= 1.0
    assert abs(float(p.scales.mean()) + 4.0) < 0.1
    np.testing.assert_allclose(p.quats.norm(dim=1).numpy(), 1.0, rtol=1e-5)
    q = serving.random_scene_tensors(1000, 3, device="cpu", sh_degree=1)
    assert all(torch.equal(a, b) for a, b in zip(p.tensors(), q.tensors()))  # seeded


def test_scene_sizes_log_uniform():
    s = serving.scene_sizes(2000, 50_000, 3_000_000, seed=1)
    assert min(s) >= 50_000 and max(s) <= 3_000_000
    logs = np.log(s)
    # uniform in log space: the median sits at the geometric mean of the bounds
    assert abs(np.median(logs) - 0.5 * (np.log(50_000) + np.log(3_000_000))) < 0.15
    assert serving.scene_sizes(32, seed=5) == serving.scene_sizes(32, seed=5)


def test_poisson_requests_rate_and_determinism():
    r1 = serving.poisson_requests(1000.0, 2.0, 32, seed=4)
    r2 = serving.poisson_requests(1000.0, 2.0, 32, seed=4)
    assert len(r1) == len(r2) and all(a.arrival == b.arrival and a.scene_id == b.scene_id for a, b in zip(r1, r2))
    assert 1800 < len(r1) < 2200
    arr = np.array([r.arrival for r in r1])
    assert np.all(np.diff(arr) > 0) and arr[-1] < 2.0
    gaps = np.diff(np.r_[0.0, arr])
    assert abs(gaps.mean() - 1e-3) < 1e-4  # exponential inter-arrival times, mean 1/rate
    res = {(r.camera.width, r.camera.height) for r in r1}
    assert res == set(serving.SERVING_RESOLUTIONS)
    for r in r1[:50]:  # cameras on the 5 m sphere
        assert abs(np.linalg.norm(r.camera.cam_pos) - 5.0) < 1e-4


def test_store_rejects_scene_over_budget():
    st = serving.SceneStore(_nbytes(1000) - 1, device="cpu")
    with pytest.raises(MemoryError):
        st.add(0, _scene(1000))
    assert len(st) == 0


def test_store_lru_eviction_order():
    st = serving.SceneStore(3 * _nbytes(1000), device="cpu")
    for i in range(5):
        st.add(i, _scene(1000, i))
    for i in (0, 1, 2):
        st.try_acquire(i)
        st.release(i)
    assert st.resident_ids() == [0, 1, 2] and st.uploads == 3 and st.evictions == 0
    st.try_acquire(0)  # touch 0: now 1 is least recently used
    st.release(0)
    st.try_acquire(3)
    st.release(3)
    assert st.resident_ids() == [2, 0, 3] and st.evictions == 1
    p = st.try_acquire(1)  # re-admission uploads the host copy again
    st.release(1)
    assert st.resident_ids() == [0, 3, 1] and st.uploads == 5
    ref = _scene(1000, 1)
    assert all(torch.equal(a, b) for a, b in zip(p.tensors(), ref.tensors()))


def test_store_never_evicts_scenes_in_use():
    st = serving.SceneStore(2 * _nbytes(1000), device="cpu")
    for i in range(3):
        st.add(i, _scene(1000, i))
    a = st.try_acquire(0)
    b = st.try_acquire(1)
    assert a is not None and b is not None
    assert st.try_acquire(2) is None  # both residents are held
    st.release(0)
    assert st.try_acquire(2) is not None  # 0 was free to evict
    assert st.resident_ids() == [1, 2]
    with pytest.raises(RuntimeError):
        st.release(0)  # over-release is an error


def test_store_reserved_bytes_count_against_budget():
    held = {"b": 0}
    st = serving.SceneStore(2 * _nbytes(1000), device="cpu", reserved=lambda: held["b"])
    for i in range(2):
        st.add(i, _scene(1000, i))
    st.try_acquire(0)
    st.release(0)
    held["b"] = _nbytes(1000)  # renderers now hold one scene's worth
    st.try_acquire(1)
    st.release(1)
    assert st.resident_ids() == [1] and st.evictions == 1


class FakeRenderer:
    """Stands in for a Context: fills each image with its request's scene id and
    width, records the batches, and takes ``delay`` seconds per call."""

    def __init__(self, log, delay=0.004):
        self.log = log
        self.delay = delay

    def device_bytes(self):
        return 0

    def render_batch(self, items, outs, stream=None):
        self.log.append(len(items))
        time.sleep(self.delay)
        for it, o in zip(items, outs):
            o.fill_(float(it.params.n) + it.camera.width / 1e4)
        return outs

    def render(self, p, cam, background, out=None):
        self.log.append(1)
        time.sleep(self.delay)
        out.fill_(float(p.n) + cam.width / 1e4)
        return out


def _requests(n_req, n_scenes, seed=0, spacing=0.0):
    rng = np.random.default_rng(seed)
    cams = [small_camera(64, 48), small_camera(32, 32), small_camera(80, 16)]
    return [serving.RenderRequest(int(rng.integers(n_scenes)), cams[int(rng.integers(3))], k * spacing, k)
            for k in range(n_req)]


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_server_serves_every_request_with_its_own_image(mode):
    st = serving.SceneStore(1 << 30, device="cpu")
    sizes = [100 + 10 * i for i in range(6)]
    for i, n in enumerate(sizes):
        st.add(i, _scene(n, i))
    log = []
    srv = serving.RenderServer(st, [0.0, 0.0, 0.0], slots=3, max_batch=8, mode=mode, keep_images=True,
                               renderer_factory=lambda: FakeRenderer(log))
    reqs = _requests(60, 6)
    res = srv.run(reqs, realtime=False)
    assert sorted(r.rid for r in res) == list(range(60))
    by = {r.rid: r for r in res}
    for q in reqs:
        img = by[q.rid].image
        assert img.shape == (q.camera.height, q.camera.width, 3)
        assert torch.all(img == float(sizes[q.scene_id]) + q.camera.width / 1e4)
    if mode == "plain":
        assert set(log) == {1}
    else:
        assert max(log) > 1 and max(log) <= 8  # requests were batched, within the cap
        assert sum(log) == 60


def test_server_continuous_batching_overlaps_slots():
    """Requests arriving while batches are in flight are taken by free workers."""
    st = serving.SceneStore(1 << 30, device="cpu")
    for i in range(4):
        st.add(i, _scene(50, i))
    active, peak, lock = [0], [0], threading.Lock()

    class Slow(FakeRenderer):
        def render_batch(self, items, outs, stream=None):
            with lock:
                active[0] += 1
                peak[0] = max(peak[0], active[0])
            try:
                return super().render_batch(items, outs, stream)
            finally:
                with lock:
                    active[0] -= 1

    log = []
    srv = serving.RenderServer(st, [0.0] * 3, slots=3, max_batch=4,
                               renderer_factory=lambda: Slow(log, delay=0.05))
    res = srv.run(_requests(40, 4, spacing=0.002), realtime=True)
    assert len(res) == 40
    assert peak[0] >= 2  # two or more batches were in flight together
    s = serving.latency_summary(res)
    assert s["requests"] == 40 and s["p99_ms"] >= s["p50_ms"] > 0 and s["mean_batch"] >= 1


def test_server_small_budget_evicts_and_completes():
    # room for two scenes plus the two workers' output arenas (4 x 64x48 pixels each)
    arena = 2 * 4 * 64 * 48 * 3 * 4
    st = serving.SceneStore(2 * _nbytes(20_000) + arena, device="cpu")
    for i in range(5):
        st.add(i, _scene(20_000, i))
    log = []
    srv = serving.RenderServer(st, [0.0] * 3, slots=2, max_batch=4, max_batch_pixels=4 * 64 * 48,
                               keep_images=True, renderer_factory=lambda: FakeRenderer(log, delay=0.001))
    reqs = _requests(50, 5, seed=3)
    res = srv.run(reqs, realtime=False)
    assert len(res) == 50 and st.evictions > 0 and st.uploads > 5
    for r in res:
        assert torch.all(r.image == 20_000.0 + r.width / 1e4)


def test_server_reports_unservable_budget():
    st = serving.SceneStore(_nbytes(200), device="cpu")
    st.add(0, _scene(200, 0))
    srv = serving.RenderServer(st, [0.0] * 3, slots=1, renderer_factory=lambda: FakeRenderer([]))
    srv.workers[0].held_bytes = 1  # the renderer's working memory leaves no room for the scene
    with pytest.raises(MemoryError):
        srv.run(_requests(3, 1), realtime=False)


def test_store_set_budget_evicts_lru_not_in_use():
    st = serving.SceneStore(4 * _nbytes(1000), device="cpu")
    for i in range(4):
        st.add(i, _scene(1000, i))
    st.try_acquire(0)  # in use: survives the shrink although least recently used
    for i in range(1, 4):
        st.try_acquire(i)
        st.release(i)
    assert st.resident_ids() == [0, 1, 2, 3]
    st.set_budget(2 * _nbytes(1000))
    assert st.resident_ids() == [0, 3] and st.evictions == 2
    st.release(0)
