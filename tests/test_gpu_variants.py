"""Rasterizer staging variants and their autotuner (needs a GPU).

The variants differ only in how many Gaussians are staged in shared memory per round
and in the backward reduction's sub-batch; images, gradients and Adam updates must be
identical, bit for bit, whichever one runs.
"""
import pytest
import torch

from msplat_street_b200 import autotune, scenes
from msplat_street_b200.backend import AdamState, BatchItem, Context, GaussianParams
from oracle_lib import Oracle
from parity_util import BACKGROUND, C1_LRS

pytestmark = pytest.mark.gpu


def _step(variant, shape=0):
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    gt = torch.from_numpy(Oracle().render(scenes.small_scene(1), cam, BACKGROUND)).cuda()
    ctx = Context(keep_grads=True)
    ctx.set_raster_variant(variant)
    ctx.set_raster_shape(shape)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    st = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx.train_step(p, adam, cam, BACKGROUND, gt, st, sync_loss=True)
    img = ctx.render(p, cam, BACKGROUND).clone()
    batch = ctx.render_batch([BatchItem(p, cam, BACKGROUND), BatchItem(p, scenes.small_camera(200, 120), BACKGROUND)])
    views = [(cam, gt), (scenes.small_camera(200, 120), gt[:120, :200].contiguous())]
    q = GaussianParams.from_numpy(g)
    ctx.train_batch(q, AdamState.zeros_like(q, C1_LRS), views, BACKGROUND)
    return [loss, img, *batch, *p.tensors(), *st, *q.tensors()]


def test_variants_give_identical_results():
    vs = autotune.raster_variants()
    assert len(vs) >= 4 and vs[0] == {"variant": 0, "fwd_batch": 128, "bwd_batch": 128, "bwd_sub": 3}
    ref = _step(0)
    for d in vs[1:]:
        got = _step(d["variant"])
        assert got[0] == ref[0], d
        for a, b in zip(got[1:], ref[1:]):
            assert torch.equal(a, b), d


def test_shapes_give_identical_results():
    """The batched forward's block shapes (16 x 16, 16 x 8, 8 x 8 pixels a block) walk
    the same 16 x 16 tile lists: batched renders and batched training steps (whose
    forward they run) match bit for bit, with every staging variant's forward round."""
    shapes = autotune.raster_shapes()
    assert [(d["w"], d["h"]) for d in shapes] == [(16, 16), (16, 8), (8, 8)]
    ref = _step(0)
    for v in (0, 3, 4):  # forward rounds of 128, 256 and 64 Gaussians
        for d in shapes[1:]:
            got = _step(v, d["shape"])
            assert got[0] == ref[0], (v, d)
            for a, b in zip(got[1:], ref[1:]):
                assert torch.equal(a, b), (v, d)


def test_shapes_on_mixed_resolutions():
    """Three views of different sizes, one not a multiple of 16, batched together."""
    from msplat_street_b200.camera import look_at, prepare_cam
    g = GaussianParams.from_numpy(scenes.small_scene(0))
    cams = [scenes.small_camera(), prepare_cam(look_at((0.8, 0.3, 2.6), (0, 0, 0)), 200, 136, 180.0, 170.0, 97.5,
                                                 70.25),
            prepare_cam(look_at((-1.2, -0.4, 2.4), (0, 0, 0)), 330, 250, 260.0, 260.0, 165.0, 125.0)]
    outs = []
    for s in (0, 1, 2):
        ctx = Context()
        ctx.set_raster_shape(s)
        outs.append([t.clone() for t in ctx.render_batch([BatchItem(g, c, BACKGROUND) for c in cams])])
        ctx.close()
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert torch.equal(a, b)


def test_bad_variant_rejected():
    with pytest.raises(ValueError):
        Context().set_raster_variant(99)
    with pytest.raises(ValueError):
        Context().set_raster_shape(3)


def test_tuner_picks_a_measured_variant():
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    ctx = Context()
    p = GaussianParams.from_numpy(g)
    res = autotune.tune_raster([ctx], lambda: ctx.render(p, cam, BACKGROUND), variants=[0, 1, 3], warmup=1, reps=3,
                               rounds=1)
    assert res["best"] in (0, 1, 3) and set(res["ms"]) == {0, 1, 3}
    assert ctx.raster_variant == res["best"]
    items = [BatchItem(p, cam, BACKGROUND), BatchItem(p, scenes.small_camera(200, 120), BACKGROUND)]
    res = autotune.tune_raster([ctx], lambda: ctx.render_batch(items), variants=[0], shapes=[0, 1, 2], warmup=1,
                               reps=3, rounds=1)
    assert set(res["ms"]) == {"0/0", "0/1", "0/2"} and ctx.raster_shape == res["best_shape"]
