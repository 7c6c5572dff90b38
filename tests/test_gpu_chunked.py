"""Depth-chunked compositing on the GPU (Context.set_chunked; the Metal backend's
path for small frames, core/metal/msplat_metal.metal:2641-3030) against the oracle's
restatement of it: the work items bit for bit, last contributors bit for bit, images
max-abs <= 1e-5, gradients relative L2 <= 1e-4 -- the one-pass path's bars. Also the
"auto" rule (fewer than 400 tiles), a frame with a prior (one pass), the
differentiable render's backward, and the one-pass result for lists of one piece."""
import numpy as np
import pytest
import torch

from msplat_street_b200 import autograd as ag
from msplat_street_b200 import scenes
from msplat_street_b200.backend import AdamState, Context, GaussianParams, PriorStep
from grad_util import oracle_param_grads
from oracle_lib import Oracle, new_adam_state, set_option
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2

pytestmark = pytest.mark.gpu

GRADS = ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")
NAMES = ("means", "scales", "quats", "dc", "rest", "opacities")


@pytest.fixture()
def oracle():
    o = Oracle("restatement")
    yield o
    set_option(o, "chunk_size", 0)


def _saturated():
    g = scenes.random_gaussians(6000, 3, log_scale_mean=-2.2)
    g.opacities[:] = 4.0  # early stops inside pieces and merged cut-offs
    return g


CASES = {
    "long_lists": (lambda: scenes.random_gaussians(20000, 3, log_scale_mean=-2.0),
                   lambda: scenes.small_camera(96, 64, 110.0)),
    "saturated": (_saturated, lambda: scenes.small_camera(100, 70, 110.0)),
    "ragged_edge": (lambda: scenes.random_gaussians(12000, 5, log_scale_mean=-2.3),
                    lambda: scenes.small_camera(83, 45, 90.0)),
}


@pytest.mark.parametrize("chunk", [64, 512])
@pytest.mark.parametrize("name", sorted(CASES))
def test_render_chunked(oracle, name, chunk):
    g, cam = CASES[name][0](), CASES[name][1]()
    set_option(oracle, "chunk_size", chunk)
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context(chunked="on", chunk_len=chunk)
    img = ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND).cpu().numpy()
    first = ctx.frame("chunk_first").cpu().numpy()
    assert np.array_equal(first, oracle.frame("chunk_first"))
    assert first[-1] > 2 * cam.tiles_x * cam.tiles_y  # several pieces per tile
    assert max_abs(img, img_o) <= IMAGE_ATOL
    assert np.array_equal(ctx.frame("final_idx").cpu().numpy(), oracle.frame("final_idx"))
    assert max_abs(ctx.frame("final_Ts").cpu().numpy(), oracle.frame("final_Ts")) <= 1e-6


@pytest.mark.parametrize("chunk", [64, 512])
@pytest.mark.parametrize("name", sorted(CASES))
def test_train_step_chunked(oracle, name, chunk):
    g, cam = CASES[name][0](), CASES[name][1]()
    set_option(oracle, "chunk_size", chunk)
    gt = np.random.default_rng(1).random((cam.height, cam.width, 3)).astype(np.float32)
    go = g.copy()
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = oracle.train_step(go, cam, BACKGROUND, gt, new_adam_state(go, C1_LRS, 1), st)
    ctx = Context(keep_grads=True, chunked="on", chunk_len=chunk)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, sync_loss=True)
    assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o))
    for key in GRADS:
        got, ref = ctx.frame(key).cpu().numpy(), oracle.frame(key)
        assert rel_l2(got, ref) <= GRAD_RTOL_L2, (key, rel_l2(got, ref))


def test_autograd_chunked(oracle):
    g, cam = CASES["long_lists"][0](), CASES["long_lists"][1]()
    set_option(oracle, "chunk_size", 512)
    gt = np.random.default_rng(2).random((cam.height, cam.width, 3)).astype(np.float32)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    oracle.train_step(g.copy(), cam, BACKGROUND, gt, new_adam_state(g, C1_LRS, 1), st)
    ref = oracle_param_grads(oracle, g, cam, 3)
    v_ref = oracle.frame("v_rendered").reshape(cam.height, cam.width, 3)
    ag.set_chunked_mode("auto")  # 24 tiles: chunked
    try:
        p = GaussianParams(*[torch.from_numpy(a).cuda().requires_grad_(True) for a in g.arrays()])
        img = ag.render(p, cam, BACKGROUND)
        assert max_abs(img.detach().cpu().numpy(), oracle.frame("out_img").reshape(img.shape)) <= IMAGE_ATOL
        img.backward(torch.from_numpy(np.ascontiguousarray(v_ref)).cuda())
        for t, b, nm in zip(p.tensors(), ref, NAMES):
            assert rel_l2(t.grad.cpu().numpy(), b) <= GRAD_RTOL_L2, (nm, rel_l2(t.grad.cpu().numpy(), b))
    finally:
        ag.set_chunked_mode("off")


def test_auto_rule_and_prior(oracle):
    g = scenes.random_gaussians(20000, 4, log_scale_mean=-2.5)
    p = GaussianParams.from_numpy(g)
    ctx = Context(chunked="auto")
    small = scenes.small_camera(320, 240, 300.0)  # 20 x 15 = 300 tiles: chunked
    ctx.render(p, small, BACKGROUND)
    assert ctx.frame("chunk_first").numel() == 301
    big = scenes.small_camera(336, 320, 300.0)  # 21 x 20 = 420 tiles: one pass
    img = ctx.render(p, big, BACKGROUND).cpu().numpy()
    assert ctx.frame("chunk_first").numel() == 0
    assert max_abs(img, oracle.render(g, big, BACKGROUND)) <= IMAGE_ATOL
    # a prior's aux rasterizer is one pass only
    ctx.set_chunked("on")
    ctx.set_prior(PriorStep(aux=True))
    ctx.render(p, small, BACKGROUND)
    assert ctx.frame("chunk_first").numel() == 0
    ctx.set_prior(None)


def test_one_piece_matches_one_pass():
    g, cam = scenes.random_gaussians(1500, 8), scenes.small_camera(80, 80, 100.0)
    p = GaussianParams.from_numpy(g)
    a = Context()
    img_a = a.render(p, cam, BACKGROUND).cpu().numpy()
    b = Context(chunked="on", chunk_len=1 << 16)
    img_b = b.render(p, cam, BACKGROUND).cpu().numpy()
    assert np.array_equal(a.frame("final_Ts").cpu().numpy(), b.frame("final_Ts").cpu().numpy())
    assert np.array_equal(a.frame("final_idx").cpu().numpy(), b.frame("final_idx").cpu().numpy())
    assert max_abs(img_a, img_b) <= 2.4e-7


def _empty_scene():
    z = np.zeros((0, 3), np.float32)
    return scenes.Gaussians(z, z, np.zeros((0, 4), np.float32), z, np.zeros((0, 15, 3), np.float32),
                            np.zeros((0, 1), np.float32))


@pytest.mark.parametrize("name", ["empty", "one_pixel", "behind_camera"])
def test_chunked_edges(oracle, name):
    """Frames with no work items (an empty scene, every Gaussian behind the camera) and
    a one-pixel frame, chunked, against the oracle's chunked restatement."""
    if name == "empty":
        g, cam = _empty_scene(), scenes.small_camera(64, 48, 80.0)
    elif name == "one_pixel":
        g, cam = scenes.random_gaussians(3000, 6, log_scale_mean=-2.0), scenes.small_camera(1, 1, 2.0)
    else:
        g = scenes.random_gaussians(500, 5)
        g.means[:, 2] += 10.0
        cam = scenes.small_camera(64, 48, 80.0)
    set_option(oracle, "chunk_size", 64)
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context(chunked="on", chunk_len=64)
    img = ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND).cpu().numpy()
    assert max_abs(img, img_o) <= IMAGE_ATOL
    assert np.array_equal(ctx.frame("chunk_first").cpu().numpy(), oracle.frame("chunk_first"))
    assert np.array_equal(ctx.frame("final_idx").cpu().numpy(), oracle.frame("final_idx"))
    if name != "one_pixel":
        assert ctx.frame("chunk_first").cpu().numpy()[-1] == 0  # no work items
        assert np.array_equal(img, np.broadcast_to(np.clip(BACKGROUND, 0, 1), img.shape))
    # and a training step through the chunked backward
    gt = np.random.default_rng(1).random((cam.height, cam.width, 3)).astype(np.float32)
    go = g.copy()
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = oracle.train_step(go, cam, BACKGROUND, gt, new_adam_state(go, C1_LRS, 1), st)
    p = GaussianParams.from_numpy(g)
    ctx2 = Context(keep_grads=True, chunked="on", chunk_len=64)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx2.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, sync_loss=True)
    assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o))
    if g.n:
        for key in GRADS:
            got, ref = ctx2.frame(key).cpu().numpy(), oracle.frame(key)
            if not np.any(ref):
                assert not np.any(got), key
            else:
                assert rel_l2(got, ref) <= GRAD_RTOL_L2, (key, rel_l2(got, ref))


def test_chunk_len_bounds():
    ctx = Context()
    with pytest.raises(ValueError):
        ctx.set_chunked("on", chunk_len=8)
    with pytest.raises(ValueError):
        ctx.set_chunked("sometimes")
