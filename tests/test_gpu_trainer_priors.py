"""Prior-guided training through the trainer on the GPU (model.cpp:548-625, 811-877):
per-camera prior maps, the learned sky, exposure and the needle cap drive the step;
depth renders, prior losses and checkpoints with the sky and exposure sections."""
import numpy as np
import pytest
import torch

from msplat_street_b200 import formats, priors, scenes
from msplat_street_b200.backend import Context, GaussianParams, PriorStep
from msplat_street_b200.camera import prepare_cam
from msplat_street_b200.trainer import Dataset, GaussianTrainer, TrainingConfig
from parity_util import BACKGROUND

pytestmark = pytest.mark.gpu

OPTS = dict(depth_weight=0.05, depth_weight_final=0.01, sky_alpha_weight=0.02, fill_weight=0.01, use_masks=True,
            learn_sky=True, sky_width=64, sky_height=16, exposure=True, max_scale_ratio=8.0)


def _setup(seed=3):
    rng = np.random.default_rng(seed)
    poses = [scenes.sphere_pose(rng, 3.0) for _ in range(4)]
    setups = [prepare_cam(p, 96, 64, 90.0, 90.0, 48.0, 32.0) for p in poses]
    ctx = Context()
    gt = GaussianParams.from_numpy(scenes.small_scene(1, 4000))
    targets, cps = [], []
    for s in setups:
        targets.append(ctx.render(gt, s, BACKGROUND).clone())
        ctx.set_prior(PriorStep(aux=True))
        ctx.render(gt, s, BACKGROUND)
        d, t = ctx.render_aux_outputs()
        depth, alpha = (x.reshape(s.height, s.width).cpu().numpy() for x in ctx.finalize_depth(d, t))
        ctx.set_prior(None)
        sky = (alpha < 0.05).astype(np.float32)  # nothing there: sky
        keep = np.ones_like(sky)
        keep[:4, :4] = 0.0
        cps.append(priors.build_camera_prior(np.where(alpha > 0.5, depth, 0.0), None, sky, keep, use_mask=True))
    views = Dataset.from_setups(setups, [None] * 4, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.uint8), poses)
    return ctx, views, targets, cps


def _trainer(ctx, ds, targets, cps):
    tr = GaussianTrainer(ds, TrainingConfig(iterations=1000, warmup_length=10 ** 6),
                         init=GaussianParams.from_numpy(scenes.small_scene(0, 3000)), context=ctx)
    tr._targets = targets
    tr.configure_priors(priors.PriorOptions(**OPTS), cps)
    return tr


def test_prior_training_steps():
    ctx, ds, targets, cps = _setup()
    tr = _trainer(ctx, ds, targets, cps)
    tex0 = tr.sky["tex"].clone()
    for _ in range(6):
        tr.step()
    losses = tr.prior_losses()
    assert losses["depth"] > 0 and losses["sky"] > 0 and losses["fill"] > 0
    assert tr.sky["steps"] == 6 and sum(tr.exposure["steps"]) == 6
    assert not torch.equal(tr.sky["tex"], tex0)
    used = [i for i, s in enumerate(tr.exposure["steps"]) if s > 0]
    ident = torch.tensor([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], dtype=torch.float32, device="cuda")
    assert all(not torch.equal(tr.exposure["params"][i], ident) for i in used)
    ls = tr.params.scales.cpu().numpy()
    srt = np.sort(ls, 1)
    assert (srt[:, 2] - srt[:, 1]).max() <= np.log(np.float32(8.0)) + 1e-5
    depth, alpha = tr.render_depth(0)
    assert depth.shape == (64, 96) and alpha.max() > 0.5 and (depth[alpha > 0.5] > 0).all()
    img = tr.render(0)  # the learned sky behind the Gaussians
    assert img.shape == (64, 96, 3) and np.isfinite(img).all()


def test_prior_checkpoint_resume(tmp_path):
    ctx, ds, targets, cps = _setup()
    a = _trainer(ctx, ds, targets, cps)
    for _ in range(4):
        a.step()
    a.save_checkpoint(str(tmp_path / "p.msplat"))
    order, rng_state = list(a._order), a._rng.bit_generator.state
    for _ in range(3):
        a.step()
    b = _trainer(Context(), ds, targets, cps)
    assert b.load_checkpoint(str(tmp_path / "p.msplat")) == 4
    b._order, b._rng.bit_generator.state = order, rng_state
    for _ in range(3):
        b.step()
    for x, y in zip(a.params.tensors(), b.params.tensors()):
        assert torch.equal(x, y)
    assert torch.equal(a.sky["tex"], b.sky["tex"]) and torch.equal(a.exposure["params"], b.exposure["params"])
    ck = formats.load_checkpoint(str(tmp_path / "p.msplat"))
    assert ck.sky["steps"] == 4 and int(np.sum(ck.exposure["steps"])) == 4
    a.save_sky(str(tmp_path / "sky.png"))
    from PIL import Image
    assert Image.open(tmp_path / "sky.png").size == (64, 16)


def test_priors_refuse_batched_steps():
    ctx, ds, targets, cps = _setup()
    tr = GaussianTrainer(ds, TrainingConfig(iterations=100), init=GaussianParams.from_numpy(scenes.small_scene(0, 500)),
                         context=ctx, views_per_step=2)
    with pytest.raises(ValueError):
        tr.configure_priors(priors.PriorOptions(**OPTS), cps)
