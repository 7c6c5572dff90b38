"""Trainer checkpoints and exports on the GPU: training resumed from a checkpoint
continues exactly as the uninterrupted run (python/bindings.cpp:372-386)."""
import numpy as np
import pytest
import torch

from msplat_street_b200 import formats, scenes
from msplat_street_b200.backend import Context, GaussianParams
from msplat_street_b200.trainer import Dataset, GaussianTrainer, TrainingConfig
from parity_util import BACKGROUND

pytestmark = pytest.mark.gpu


def _trainer():
    rng = np.random.default_rng(3)
    poses = [scenes.sphere_pose(rng, 3.0) for _ in range(4)]
    from msplat_street_b200.camera import prepare_cam
    setups = [prepare_cam(p, 96, 64, 90.0, 90.0, 48.0, 32.0) for p in poses]
    ctx = Context()
    gt = GaussianParams.from_numpy(scenes.small_scene(1, 4000))
    targets = [ctx.render(gt, s, BACKGROUND).clone() for s in setups]
    ds = Dataset.from_setups(setups, [None] * 4, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.uint8), poses)
    tr = GaussianTrainer(ds, TrainingConfig(iterations=1000, warmup_length=10 ** 6),
                         init=GaussianParams.from_numpy(scenes.small_scene(0, 3000)), context=ctx)
    tr._targets = targets
    return tr


def test_resume_from_checkpoint_continues_the_run(tmp_path):
    a = _trainer()
    for _ in range(5):
        a.step()
    a.save_checkpoint(str(tmp_path / "c.msplat"))
    order = list(a._order)
    rng_state = a._rng.bit_generator.state
    for _ in range(3):
        a.step()
    b = _trainer()
    assert b.load_checkpoint(str(tmp_path / "c.msplat")) == 5
    b._order, b._rng.bit_generator.state = order, rng_state  # the camera schedule is not part of a checkpoint
    for _ in range(3):
        b.step()
    for x, y in zip(a.params.tensors(), b.params.tensors()):
        assert torch.equal(x, y)
    ck = formats.load_checkpoint(str(tmp_path / "c.msplat"))
    assert ck.adam_step == 5 and ck.num_active == 3000


def test_exports(tmp_path):
    tr = _trainer()
    tr.step()
    tr.export_ply(str(tmp_path / "s.ply"))
    tr.export_splat(str(tmp_path / "s.splat"))
    params, _ = formats.load_ply(str(tmp_path / "s.ply"))
    for x, y in zip(params, tr.params.numpy()):
        assert np.array_equal(x, y.reshape(x.shape))
    assert formats.read_splat(str(tmp_path / "s.splat")).shape == (3000,)
    rgba = tr.render_rgba8(0)
    assert rgba.shape == (64, 96, 4) and rgba.dtype == np.uint8 and (rgba[..., 3] == 255).all()
    psnr, ssim, l1 = tr.evaluate(0)
    assert np.isfinite(psnr) and 0 < ssim <= 1 and l1 >= 0


def test_read_loss_async_matches_the_synchronous_loss():
    a, b = _trainer(), _trainer()
    pinned = torch.zeros(1, dtype=torch.float32).pin_memory()
    for _ in range(3):
        a.step(sync_loss=True)
        b.step()
        ev = b.ctx.read_loss_async(pinned)
        ev.synchronize()
        assert float(pinned[0]) == a.last_loss
    with pytest.raises(ValueError):
        b.ctx.read_loss_async(torch.zeros(1))  # not pinned


def test_trainer_follows_the_resolution_schedule_and_the_oracle():
    """GaussianTrainer's own steps against the oracle fed with the reference Model's
    host values (prepareCam at the step's level, the target's area-downsampled
    pyramid level, the Adam scalars, the means LR decay, the SH ramp), over steps that
    cross two level changes and two SH-degree changes. Odd sizes (97 x 61) exercise
    the levels' integer division and per-axis intrinsics ratios."""
    from msplat_street_b200.backend import adam_step_scalars
    from msplat_street_b200.camera import prepare_cam, schedule_downscale_factor
    from msplat_street_b200.trainer import LR_INIT, means_lr, sh_degrees_to_use
    from oracle_lib import Oracle
    from parity_util import GRAD_RTOL_L2, rel_l2

    rng = np.random.default_rng(5)
    poses = [scenes.sphere_pose(rng, 3.0) for _ in range(3)]
    setups = [prepare_cam(p, 97, 61, 90.0, 88.0, 48.3, 30.2) for p in poses]
    ctx = Context()
    gt = GaussianParams.from_numpy(scenes.small_scene(1, 3000))
    targets = [ctx.render(gt, s, BACKGROUND).clone() for s in setups]
    ds = Dataset.from_setups(setups, [None] * 3, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.uint8), poses)
    cfg = TrainingConfig(iterations=40, warmup_length=10 ** 6, num_downscales=2, resolution_schedule=3,
                         sh_degree_interval=2)
    init = scenes.small_scene(0, 2000)
    tr = GaussianTrainer(ds, cfg, init=GaussianParams.from_numpy(init), context=ctx)
    tr._targets = targets
    ora = Oracle()
    go = init.copy()
    m1 = [np.zeros_like(a) for a in go.arrays()]
    m2 = [np.zeros_like(a) for a in go.arrays()]
    st = {k: np.zeros(go.n, np.float32) for k in ("vis", "gn", "ms")}
    lrs = list(LR_INIT)
    full = [t.cpu().numpy() for t in targets]
    seen = set()
    for step in range(1, 9):
        tr.step()
        (ci,) = tr.last_views
        factor = schedule_downscale_factor(step, cfg.num_downscales, cfg.resolution_schedule)
        s = prepare_cam(poses[ci], 97, 61, 90.0, 88.0, 48.3, 30.2, factor=factor)
        seen.add((factor, s.width, s.height))
        assert (tr.last_width, tr.last_height) == (s.width, s.height)
        tgt = full[ci] if factor == 1 else ora.resize_area(full[ci], s.width, s.height)
        if factor > 1:
            assert np.array_equal(tr.target_at(ci, factor).cpu().numpy(), tgt)
        ss, b2 = adam_step_scalars(lrs, step)
        ad = {"m1": m1, "m2": m2, "step_sizes": list(ss), "bc2": list(b2), "beta1": 0.9, "beta2": 0.999,
              "eps": 1e-8}
        ora.train_step(go, s, BACKGROUND, tgt, ad, st, degrees_to_use=sh_degrees_to_use(step, cfg))
        lrs[0] = means_lr(step, cfg.iterations)
        assert np.float32(tr.lrs[0]) == np.float32(lrs[0])
        for a, b in zip(tr.params.numpy(), go.arrays()):
            assert rel_l2(a, b) <= GRAD_RTOL_L2, step
    assert seen == {(4, 24, 15), (2, 48, 30), (1, 97, 61)}
