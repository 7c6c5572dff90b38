"""Batched multi-view rendering and the render server on the GPU.

Every view of a batch must equal, bit for bit, the single-view msplat_render of the
same scene and camera (which the parity tests tie to the oracle), whatever else is in
the batch and in whatever order; the server must return for every request the image
that request gets when rendered alone.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import scenes, serving
from msplat_street_b200.backend import BatchItem, Context, GaussianParams
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle
from parity_util import BACKGROUND

pytestmark = pytest.mark.gpu


def _dev(g):
    return GaussianParams.from_numpy(g)


def _empty_scene():
    z = np.zeros((0, 3), np.float32)
    return GaussianParams.from_numpy(scenes.Gaussians(z, z, np.zeros((0, 4), np.float32), z,
                                                      np.zeros((0, 15, 3), np.float32), np.zeros((0, 1), np.float32)))


def _items():
    rng = np.random.default_rng(21)
    s0 = _dev(scenes.small_scene(0))                                   # 10k, SH degree 3
    s1 = _dev(scenes.random_gaussians(3000, 4, sh_degree=1))           # SH degree 1
    s2 = _dev(scenes.random_gaussians(20_000, 5, sh_degree=0))         # no higher SH
    s3 = _empty_scene()
    side = prepare_cam(look_at((0.3, 0.2, 2.5), (0, 0, 0)), 200, 136, 180.0, 170.0, 97.5, 70.25)
    bg2 = np.array([0.1, 0.2, 0.3], np.float32)
    return [
        BatchItem(s0, scenes.small_camera(), BACKGROUND),
        BatchItem(s1, side, bg2),
        BatchItem(s0, scenes.sphere_camera(rng, 512, 512, radius=3.0), BACKGROUND),
        BatchItem(s3, scenes.small_camera(48, 40), bg2),
        BatchItem(s2, scenes.sphere_camera(rng, 1280, 720, radius=3.0), BACKGROUND),
        BatchItem(s0, scenes.small_camera(256, 256), BACKGROUND, degrees_to_use=1),
        BatchItem(s2, scenes.small_camera(33, 17, f=40.0), bg2),
    ]


def _alone(ctx, it):
    return ctx.render(it.params, it.camera, it.background, degrees_to_use=it.degrees_to_use).clone()


def test_batch_equals_single_view_renders():
    ctx = Context()
    items = _items()
    alone = [_alone(ctx, it) for it in items]
    got = ctx.render_batch(items)
    torch.cuda.synchronize()
    for k, (a, b) in enumerate(zip(alone, got)):
        assert torch.equal(a, b), f"view {k}: max |diff| {float((a - b).abs().max())}"
    # the empty scene shows its background everywhere
    assert torch.equal(got[3], torch.tensor(items[3].background, device="cuda").expand_as(got[3]))


def test_batch_is_independent_of_order_and_company():
    ctx = Context()
    items = _items()
    ref = [t.clone() for t in ctx.render_batch(items)]
    perm = [4, 0, 6, 2, 5, 1, 3]
    got = ctx.render_batch([items[p] for p in perm])
    for j, p in enumerate(perm):
        assert torch.equal(got[j], ref[p])
    for k in (0, 4):  # one view alone in a batch of one
        assert torch.equal(ctx.render_batch([items[k]])[0], ref[k])
    # many copies of one view in one batch
    many = ctx.render_batch([items[1]] * 9)
    for t in many:
        assert torch.equal(t, ref[1])


def test_batch_view_matches_oracle():
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    ctx = Context()
    out = ctx.render_batch([BatchItem(_dev(g), cam, BACKGROUND),
                            BatchItem(_dev(scenes.small_scene(1)), cam, BACKGROUND)])
    ref = Oracle().render(g, cam, BACKGROUND)
    assert float(np.abs(out[0].cpu().numpy() - ref).max()) <= 1e-5


def test_batch_writes_into_given_outputs_and_rejects_bad_ones():
    ctx = Context()
    it = _items()[0]
    out = torch.full((256, 256, 3), -1.0, device="cuda")
    r = ctx.render_batch([it], outs=[out])
    assert r[0] is out and float(out.min()) >= 0.0
    with pytest.raises(ValueError):
        ctx.render_batch([it], outs=[torch.empty((255, 256, 3), device="cuda")])


def _server_scenes(store, sizes, seed=40):
    for i, n in enumerate(sizes):
        store.add(i, serving.random_scene_tensors(n, seed + i), resident=True)


def _check_alone(results, reqs, store):
    ctx = Context()
    by = {r.rid: r for r in results}
    for q in reqs:
        p = store.try_acquire(q.scene_id)
        try:
            a = ctx.render(p, q.camera, BACKGROUND)
        finally:
            store.release(q.scene_id)
        assert torch.equal(by[q.rid].image, a), f"request {q.rid} differs from its render alone"


def test_server_results_equal_alone_renders():
    store = serving.SceneStore(8 << 30)
    _server_scenes(store, [60_000, 150_000, 20_000, 300_000])
    reqs = serving.poisson_requests(2000.0, 0.05, 4, seed=8, resolutions=((512, 512), (1280, 720), (320, 200)),
                                    radius=4.0)
    srv = serving.RenderServer(store, BACKGROUND, slots=3, max_batch=8, keep_images=True)
    res = srv.run(reqs, realtime=True)
    assert len(res) == len(reqs) and max(r.batch_size for r in res) > 1
    _check_alone(res, reqs, store)
    plain = serving.RenderServer(store, BACKGROUND, mode="plain", keep_images=True)
    _check_alone(plain.run(reqs[:10], realtime=False), reqs[:10], store)
    srv.close()
    plain.close()


def test_server_small_budget_lru():
    sizes = [300_000, 340_000, 380_000, 320_000, 360_000]
    per = [n * 59 * 4 for n in sizes]
    store = serving.SceneStore(64 << 30)
    for i, n in enumerate(sizes):
        store.add(i, serving.random_scene_tensors(n, 40 + i), resident=False)
    reqs = serving.poisson_requests(1000.0, 0.05, 5, seed=9, resolutions=((256, 256), (200, 120)), radius=4.0)
    srv = serving.RenderServer(store, BACKGROUND, slots=1, max_batch=2, max_batch_pixels=2 * 256 * 256,
                               keep_images=True)
    srv.run(reqs[:8], realtime=False)  # sizes the render context's caches
    # room for the two largest scenes and the renderer's working memory, not for five scenes
    store.set_budget(int(sum(sorted(per)[-2:]) + 1.5 * srv.reserved_bytes()))
    assert store.resident_bytes <= store.budget
    uploads = store.uploads
    res = srv.run(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert store.evictions > 0 and store.uploads > uploads
    assert store.resident_bytes <= store.budget
    _check_alone(res, reqs, store)
    srv.close()
