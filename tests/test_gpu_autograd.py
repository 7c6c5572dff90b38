"""The differentiable path (msplat_street_b200.autograd) on the GPU.

Case 1: 64 Gaussians, 32x32, every parameter against float64 central finite
differences (h = 1e-4, tests/golden/fd_smooth.npz) with the reference's gradient-check
criterion, and against the CPU oracle's gradients.
Case 2: 200,000 Gaussians at 1024x768 against the oracle: image, loss, and every
parameter gradient (relative L2 <= 1e-4).
"""
import os

import numpy as np
import pytest
import torch

from msplat_street_b200 import autograd as ag
from msplat_street_b200 import scenes
from msplat_street_b200.backend import GaussianParams
from grad_util import fd_agreement, oracle_param_grads
from oracle_lib import Oracle, new_adam_state
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2
from smooth_scenes import smooth_scene

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ("means", "scales", "quats", "dc", "rest", "opacities")


def _leaf_params(g):
    return GaussianParams(*[torch.from_numpy(a).cuda().requires_grad_(True) for a in g.arrays()])


def _autograd_grads(g, cam, gt, ssim_weight=0.2):
    p = _leaf_params(g)
    img = ag.render(p, cam, BACKGROUND)
    loss = ag.ssim_l1_loss(img, torch.from_numpy(gt).cuda(), ssim_weight)
    loss.backward()
    return [t.grad.cpu().numpy() for t in p.tensors()], float(loss.detach()), img.detach().cpu().numpy()


@pytest.mark.parametrize("view_dependent", [False, True])
def test_autograd_matches_finite_differences(view_dependent):
    g, cam, gt = smooth_scene(view_dependent=view_dependent)
    fx = dict(np.load(os.path.join(GOLDEN, "fd_smooth.npz")))
    tag = "vd" if view_dependent else "flat"
    fd = [fx[f"{tag}_{k}"] for k in NAMES]
    grads, loss, _ = _autograd_grads(g, cam, gt)
    skip = (0,) if view_dependent else ()
    bad, checked, cos = fd_agreement(grads, fd, skip=skip)
    assert bad == 0 and cos > 0.9999, (bad, checked, cos)
    # and the CPU oracle's gradients on the same state
    ora = Oracle("restatement")
    ad = new_adam_state(g, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = ora.train_step(g.copy(), cam, BACKGROUND, gt, ad, st)
    assert abs(loss - loss_o) <= 1e-6
    for a, b, nm in zip(grads, oracle_param_grads(ora, g, cam, 3), NAMES):
        assert rel_l2(a, b) <= GRAD_RTOL_L2, (nm, rel_l2(a, b))


def test_autograd_case2_200k_1024x768():
    g = scenes.random_gaussians(200_000, 21)
    cam = scenes.small_camera(1024, 768, 1000.0, 3.0)
    ora = Oracle("restatement")
    gt = ora.render(scenes.random_gaussians(200_000, 22), cam, BACKGROUND)
    ad = new_adam_state(g, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = ora.train_step(g.copy(), cam, BACKGROUND, gt, ad, st)
    ref_grads = oracle_param_grads(ora, g, cam, 3)
    v_ref = ora.frame("v_rendered").reshape(cam.height, cam.width, 3)
    img_o = ora.frame("out_img").reshape(cam.height, cam.width, 3)

    # the backward pipeline alone: our image's backward fed the oracle's dL/d(image)
    p = _leaf_params(g)
    img = ag.render(p, cam, BACKGROUND)
    assert max_abs(img.detach().cpu().numpy(), img_o) <= IMAGE_ATOL
    img.backward(torch.from_numpy(np.ascontiguousarray(v_ref)).cuda())
    for t, b, nm in zip(p.tensors(), ref_grads, NAMES):
        assert rel_l2(t.grad.cpu().numpy(), b) <= GRAD_RTOL_L2, (nm, rel_l2(t.grad.cpu().numpy(), b))

    # the whole loss through autograd
    grads, loss, _ = _autograd_grads(g, cam, gt)
    assert abs(loss - loss_o) <= 1e-6
    for a, b, nm in zip(grads, ref_grads, NAMES):
        assert rel_l2(a, b) <= GRAD_RTOL_L2, (nm, rel_l2(a, b))


def test_autograd_two_views_accumulate():
    """Two renders alive in one graph: the summed loss's gradient equals the sum of the
    two single-view gradients."""
    g = scenes.random_gaussians(5000, 3)
    cams = [scenes.small_camera(128, 96, 150.0, 3.0), scenes.small_camera(96, 128, 140.0, 2.6)]
    ora = Oracle("restatement")
    gts = [torch.from_numpy(ora.render(scenes.random_gaussians(5000, 4), c, BACKGROUND)).cuda() for c in cams]
    p = _leaf_params(g)
    loss = sum(ag.ssim_l1_loss(ag.render(p, c, BACKGROUND), t) for c, t in zip(cams, gts))
    loss.backward()
    together = [t.grad.clone() for t in p.tensors()]
    single = [torch.zeros_like(t) for t in p.tensors()]
    for c, t in zip(cams, gts):
        q = _leaf_params(g)
        ag.ssim_l1_loss(ag.render(q, c, BACKGROUND), t).backward()
        for s, x in zip(single, q.tensors()):
            s += x.grad
    for a, b in zip(together, single):
        assert torch.allclose(a, b, rtol=1e-5, atol=1e-9)


def test_render_without_grad_matches_render():
    g = scenes.random_gaussians(3000, 8)
    cam = scenes.small_camera(100, 70, 120.0)
    p = GaussianParams.from_numpy(g)
    with torch.no_grad():
        a = ag.render(p, cam, BACKGROUND)
    b = Oracle("restatement").render(g, cam, BACKGROUND)
    assert max_abs(a.cpu().numpy(), b) <= IMAGE_ATOL


@pytest.mark.parametrize("capacity", [256, 4])
def test_autograd_stored_transmittance(capacity):
    """Stored transmittance (capacity 256: every pixel stored; 4: most pixels overflow
    and fall back to division) gives the oracle's gradients like the default mode."""
    g = scenes.random_gaussians(40_000, 31)
    cam = scenes.small_camera(320, 240, 310.0, 3.0)
    ora = Oracle("restatement")
    gt = ora.render(scenes.random_gaussians(40_000, 32), cam, BACKGROUND)
    ad = new_adam_state(g, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    ora.train_step(g.copy(), cam, BACKGROUND, gt, ad, st)
    ref_grads = oracle_param_grads(ora, g, cam, 3)
    v_ref = torch.from_numpy(np.ascontiguousarray(ora.frame("v_rendered").reshape(cam.height, cam.width, 3))).cuda()
    ag.set_transmittance_mode("store", capacity)
    try:
        p = _leaf_params(g)
        img = ag.render(p, cam, BACKGROUND)
        img.backward(v_ref)
    finally:
        ag.set_transmittance_mode("recompute")
    for t, b, nm in zip(p.tensors(), ref_grads, NAMES):
        assert rel_l2(t.grad.cpu().numpy(), b) <= GRAD_RTOL_L2, (nm, capacity, rel_l2(t.grad.cpu().numpy(), b))
