"""CUDA path vs the CPU oracle on the same seeded inputs (needs a GPU).

Bar: tile keys, sorted order, tile ranges, radii, final_idx bit-exact; rendered
images max-abs <= 1e-5; gradients relative L2 <= 1e-4; all arithmetic FP32.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import scenes
from msplat_street_b200.backend import AdamState, Context, GaussianParams
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle, new_adam_state
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2, splat_fields

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Oracle("restatement")


def _cases():
    # (name, scene, camera): the small plain config plus odd sizes, a close camera
    # with huge splats, and SH degrees 0..3
    yield "c1", scenes.small_scene(0), scenes.small_camera()
    yield "odd", scenes.random_gaussians(3000, 5), prepare_cam(look_at((0.4, -0.3, 2.5), (0, 0, 0)), 203, 117, 180.0,
                                                               170.0, 101.0, 60.5)
    yield "close", scenes.random_gaussians(2000, 6, log_scale_mean=-2.0), scenes.small_camera(96, 80, 120.0, 1.6)
    for d in range(3):
        yield f"deg{d}", scenes.random_gaussians(1500, 7 + d, sh_degree=d), scenes.small_camera(128, 96, 150.0)


@pytest.mark.parametrize("case", list(range(6)))
def test_forward_bit_exact(oracle, case):
    name, g, cam = list(_cases())[case]
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context()
    p = GaussianParams.from_numpy(g)
    img = ctx.render(p, cam, BACKGROUND).cpu().numpy()
    radii_o = oracle.frame("radii")
    radii = ctx.frame("radii").cpu().numpy()
    assert np.array_equal(radii, radii_o), name
    vis = radii_o > 0
    sp = splat_fields(ctx.frame("splats").cpu().numpy())
    for key, k in (("xys", 2), ("conics", 3), ("colors", 3), ("depths", 1)):
        ref = oracle.frame(key).reshape(g.n, k)[vis]
        got = sp[key].reshape(g.n, k)[vis]
        assert np.array_equal(got, ref), (name, key, max_abs(got, ref))
    for key in ("tile_start", "tile_end", "isect_gid", "final_idx"):
        assert np.array_equal(ctx.frame(key).cpu().numpy(), oracle.frame(key)), (name, key)
    assert max_abs(ctx.frame("final_Ts").cpu().numpy(), oracle.frame("final_Ts")) <= IMAGE_ATOL
    assert max_abs(img, img_o) <= IMAGE_ATOL, (name, max_abs(img, img_o))


def _one_step(oracle, g, cam, gt, ssim_weight=0.2):
    go = g.copy()
    ad = new_adam_state(go, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = oracle.train_step(go, cam, BACKGROUND, gt, ad, st, ssim_weight=ssim_weight)
    ctx = Context(keep_grads=True)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, ssim_weight=ssim_weight,
                          sync_loss=True)
    return ctx, p, adam, stats, loss, go, ad, st, loss_o


@pytest.mark.parametrize("ssim_weight", [0.0, 0.2, 1.0])
def test_train_step_gradients(oracle, ssim_weight):
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    gt = oracle.render(scenes.small_scene(1), cam, BACKGROUND)
    ctx, p, adam, stats, loss, go, ad, st, loss_o = _one_step(oracle, g, cam, gt, ssim_weight)
    assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o)), (loss, loss_o)
    assert max_abs(ctx.frame("v_rendered").cpu().numpy(), oracle.frame("v_rendered")) == 0.0
    for key in ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat"):
        got = ctx.frame(key).cpu().numpy()
        ref = oracle.frame(key)
        assert rel_l2(got, ref) <= GRAD_RTOL_L2, (key, rel_l2(got, ref))
    # parameter updates of the Adam step (the first step moves each element by about
    # +-lr whatever the gradient's size, so updates are compared as vectors)
    for before, gpu, ref, nm in zip(g.arrays(), p.numpy(), go.arrays(), ("means", "scales", "quats", "dc", "rest",
                                                                            "opacities")):
        assert rel_l2(gpu - before, ref - before) <= 1e-3, nm
    for k, t in zip(("vis", "gn", "ms"), stats):
        assert rel_l2(t.cpu().numpy(), st[k]) <= GRAD_RTOL_L2, k


def test_hundred_steps_c1(oracle):
    """Config: 10k Gaussians, 256x256, 100 Adam steps of L1 + 0.2 (1 - SSIM); image,
    loss and every gradient compared with the oracle at each step."""
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    gt = oracle.render(scenes.small_scene(1), cam, BACKGROUND)
    go = g.copy()
    m1 = [np.zeros_like(a) for a in go.arrays()]
    m2 = [np.zeros_like(a) for a in go.arrays()]
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    ctx = Context(keep_grads=True)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    gt_t = torch.from_numpy(gt).cuda()
    worst = {"img": 0.0, "grad": 0.0, "loss": 0.0}
    for step in range(1, 101):
        ad = new_adam_state(go, C1_LRS, step)
        ad["m1"], ad["m2"] = m1, m2
        loss_o = oracle.train_step(go, cam, BACKGROUND, gt, ad, st)
        loss = ctx.train_step(p, adam, cam, BACKGROUND, gt_t, stats, sync_loss=True)
        worst["loss"] = max(worst["loss"], abs(loss - loss_o))
        worst["img"] = max(worst["img"], max_abs(ctx.frame("out_img").cpu().numpy(), oracle.frame("out_img")))
        for key in ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat"):
            worst["grad"] = max(worst["grad"], rel_l2(ctx.frame(key).cpu().numpy(), oracle.frame(key)))
    print("worst over 100 steps:", worst)
    assert worst["img"] <= IMAGE_ATOL
    assert worst["grad"] <= GRAD_RTOL_L2
    assert worst["loss"] <= 1e-5
