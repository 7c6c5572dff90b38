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


def _step(variant):
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    gt = torch.from_numpy(Oracle().render(scenes.small_scene(1), cam, BACKGROUND)).cuda()
    ctx = Context(keep_grads=True)
    ctx.set_raster_variant(variant)
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


def test_bad_variant_rejected():
    with pytest.raises(ValueError):
        Context().set_raster_variant(99)


def test_tuner_picks_a_measured_variant():
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    ctx = Context()
    p = GaussianParams.from_numpy(g)
    res = autotune.tune_raster([ctx], lambda: ctx.render(p, cam, BACKGROUND), variants=[0, 1, 3], warmup=1, reps=3,
                               rounds=1)
    assert res["best"] in (0, 1, 3) and set(res["ms"]) == {0, 1, 3}
    assert ctx.raster_variant == res["best"]
