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
