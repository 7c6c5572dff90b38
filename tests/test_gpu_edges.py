"""Edge cases of the plain path against the CPU oracle (needs a GPU): an empty scene,
every Gaussian behind the camera, one-pixel and one-row images, a Gaussian covering
the whole image, saturated opacities (alpha capped at 0.999, early termination), and
SH degree 0. Bars as the plain parity tests: integer data bit-exact, images max-abs
<= 1e-5, gradients relative L2 <= 1e-4."""
import numpy as np
import pytest
import torch

from msplat_street_b200 import scenes
from msplat_street_b200.backend import AdamState, Context, GaussianParams
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle, new_adam_state
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2

pytestmark = pytest.mark.gpu

GRAD_KEYS = ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")


@pytest.fixture(scope="module")
def oracle():
    return Oracle("restatement")


def _empty(deg=3):
    z = np.zeros((0, 3), np.float32)
    return scenes.Gaussians(z, z, np.zeros((0, 4), np.float32), z, np.zeros((0, (deg + 1) ** 2 - 1, 3), np.float32),
                            np.zeros((0, 1), np.float32))


def _saturated(n=800, seed=3):
    g = scenes.random_gaussians(n, seed, log_scale_mean=-2.5)
    g.opacities[:] = 8.0  # sigmoid ~ 0.9997: alpha capped at 0.999, pixels terminate early
    return g


def _huge(seed=4):
    g = scenes.random_gaussians(50, seed, log_scale_mean=-4.0)
    g.means[0] = 0.0
    g.scales[0] = np.log(3.0)  # wider than the whole view
    g.opacities[0] = -1.0
    return g


def _behind(n=500, seed=5):
    g = scenes.random_gaussians(n, seed)
    g.means[:, 2] += 10.0  # the camera sits at z = 3 looking down -z: everything behind it
    return g


CASES = {
    "empty": (_empty, lambda: scenes.small_camera(64, 48, 80.0)),
    "behind_camera": (_behind, lambda: scenes.small_camera(64, 48, 80.0)),
    "one_pixel": (lambda: scenes.random_gaussians(300, 6, log_scale_mean=-2.0), lambda: scenes.small_camera(1, 1, 2.0)),
    "one_row": (lambda: scenes.random_gaussians(400, 7, log_scale_mean=-2.5), lambda: scenes.small_camera(37, 1, 30.0)),
    "huge": (_huge, lambda: prepare_cam(look_at((0.2, 0.1, 2.0), (0, 0, 0)), 80, 60, 70.0, 70.0, 40.0, 30.0)),
    "saturated": (_saturated, lambda: scenes.small_camera(96, 64, 110.0)),
    "sh_degree_0": (lambda: scenes.random_gaussians(1500, 8, sh_degree=0), lambda: scenes.small_camera(80, 80, 100.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_render_edge(oracle, name):
    make_g, make_cam = CASES[name]
    g, cam = make_g(), make_cam()
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context()
    img = ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND).cpu().numpy()
    assert max_abs(img, img_o) <= IMAGE_ATOL
    for key in ("tile_start", "tile_end", "final_idx"):
        assert np.array_equal(ctx.frame(key).cpu().numpy(), oracle.frame(key)), key
    if g.n:
        assert np.array_equal(ctx.frame("radii").cpu().numpy(), oracle.frame("radii"))
    if name in ("empty", "behind_camera"):
        assert np.array_equal(img, np.broadcast_to(np.clip(BACKGROUND, 0, 1), img.shape))
        assert ctx.num_isects() == 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_train_step_edge(oracle, name):
    make_g, make_cam = CASES[name]
    g, cam = make_g(), make_cam()
    gt = np.random.default_rng(1).random((cam.height, cam.width, 3)).astype(np.float32)
    go = g.copy()
    ad = new_adam_state(go, C1_LRS, 1)
    ad["m1"] = [np.full_like(a, 0.01) for a in g.arrays()]  # nonzero moments: every Gaussian's decay shows
    ad["m2"] = [np.full_like(a, 0.02) for a in g.arrays()]
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = oracle.train_step(go, cam, BACKGROUND, gt, ad, st)
    ctx = Context(keep_grads=True)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    for t in adam.exp_avg:
        t.fill_(0.01)
    for t in adam.exp_avg_sq:
        t.fill_(0.02)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, sync_loss=True)
    assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o)), (loss, loss_o)
    if g.n == 0:
        return
    for key in GRAD_KEYS:
        got, ref = ctx.frame(key).cpu().numpy(), oracle.frame(key)
        if not np.any(ref):
            assert not np.any(got), key  # nothing visible: exactly zero
        else:
            assert rel_l2(got, ref) <= GRAD_RTOL_L2, (key, rel_l2(got, ref))
    # the Adam step: updates compared as vectors (each element moves by about its
    # learning rate whatever its gradient), moments and statistics likewise
    for before, gpu, ref, nm in zip(g.arrays(), p.numpy(), go.arrays(),
                                    ("means", "scales", "quats", "dc", "rest", "opacities")):
        d_gpu, d_ref = gpu.reshape(ref.shape) - before, ref - before
        if np.any(d_ref):
            assert rel_l2(d_gpu, d_ref) <= 1e-3, nm
        else:
            assert not np.any(d_gpu), nm
    for gpu, ref in zip(adam.exp_avg + adam.exp_avg_sq, ad["m1"] + ad["m2"]):
        assert rel_l2(gpu.cpu().numpy().reshape(ref.shape), ref) <= GRAD_RTOL_L2
    assert np.array_equal(stats[0].cpu().numpy(), st["vis"])
    assert rel_l2(stats[1].cpu().numpy(), st["gn"]) <= GRAD_RTOL_L2
    assert np.array_equal(stats[2].cpu().numpy(), st["ms"])
