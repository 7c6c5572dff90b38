"""Parity at the benchmarked scales (needs a GPU).

1. The street workload the benchmark times: the 500,000-Gaussian ground-truth scene in
   its 20 x 4 x 20 m box, cameras inside it at 1024 x 512, training from 100,000
   jittered ground-truth means with kNN-initialised scales. The ground-truth render,
   the initialisation, three training steps (each from the oracle's state, so every
   step is compared from identical inputs) and one densification with the statistics
   those steps accumulated are compared with the oracle at the parity bars: tile
   ranges, sorted ids, radii and last contributors bit-exact, images 1e-5, loss 1e-6
   relative, gradients and Adam moments 1e-4 relative L2 (the quaternion gradient of
   the isotropic initial Gaussians, zero in exact arithmetic, against the scale
   gradient's norm), densified counts exact.
2. A render of the serving distribution at 1920 x 1080 with 1.5 M Gaussians.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import scenes, workloads
from msplat_street_b200.backend import AdamState, Context, GaussianParams
from msplat_street_b200.camera import logf
from msplat_street_b200.trainer import LR_INIT
from oracle_lib import Oracle, new_adam_state
from parity_util import BACKGROUND, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2

pytestmark = pytest.mark.gpu

GRAD_KEYS = ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")
INT_KEYS = ("radii", "tile_start", "tile_end", "isect_gid", "final_idx")


@pytest.fixture(scope="module")
def oracle():
    return Oracle("restatement")


def _ulps(a, b):
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-2 ** 31) - ia, ia)
    ib = np.where(ib < 0, np.int64(-2 ** 31) - ib, ib)
    return np.abs(ia - ib)


def _check_frame(ctx, oracle, img_gpu, img_ref, what):
    for key in INT_KEYS:
        assert np.array_equal(ctx.frame(key).cpu().numpy(), oracle.frame(key)), (what, key)
    assert max_abs(img_gpu, img_ref) <= IMAGE_ATOL, (what, max_abs(img_gpu, img_ref))
    assert max_abs(ctx.frame("final_Ts").cpu().numpy(), oracle.frame("final_Ts")) <= IMAGE_ATOL, what


def test_street_scene_render_init_steps_and_densify(oracle):
    gt, poses, setups = workloads.street_views()
    ctx = Context(keep_grads=True)
    # the ground truth's own renders are the targets; the first one against the oracle
    pg = GaussianParams.from_numpy(gt)
    targets = [ctx.render(pg, s, BACKGROUND).clone() for s in setups[:3]]
    _check_frame(ctx, oracle, targets[2].cpu().numpy(), oracle.render(gt, setups[2], BACKGROUND), "ground truth")
    del pg

    # the training start: exact 3-NN scales, random rotations, DC from the colours
    pts, rgb = scenes.jittered_init_points(gt, workloads.STREET_INIT_N, seed=3)
    logit = float(logf(np.float32(0.1) / np.float32(0.9)))
    p = ctx.init_gaussians(torch.from_numpy(pts).cuda(), torch.from_numpy(rgb), seed=42, opacity_logit=logit)
    s_o, q_o, d_o, o_o = oracle.init_gaussians(pts, rgb, 42, logit)
    # log / sin / cos in double, rounded once: within 2 ulps of glibc's float functions
    assert _ulps(p.scales.cpu().numpy(), s_o).max() <= 2 and _ulps(p.quats.cpu().numpy(), q_o).max() <= 2
    assert np.array_equal(p.features_dc.cpu().numpy(), d_o) and np.array_equal(p.opacities.cpu().numpy(), o_o)

    go = scenes.Gaussians(*[a.copy() for a in p.numpy()])
    n = go.n
    m1 = [np.zeros_like(a) for a in go.arrays()]
    m2 = [np.zeros_like(a) for a in go.arrays()]
    st = {k: np.zeros(n, np.float32) for k in ("vis", "gn", "ms")}
    adam = AdamState.zeros_like(p, LR_INIT)
    stats = tuple(torch.zeros(n, device="cuda") for _ in range(3))
    for step in (1, 2, 3):
        cam, tgt = setups[step - 1], targets[step - 1]
        # both sides start the step from the oracle's state
        for t, a in zip(p.tensors(), go.arrays()):
            t.copy_(torch.from_numpy(a))
        for t, a in zip(adam.exp_avg, m1):
            t.copy_(torch.from_numpy(a))
        for t, a in zip(adam.exp_avg_sq, m2):
            t.copy_(torch.from_numpy(a))
        for t, k in zip(stats, ("vis", "gn", "ms")):
            t.copy_(torch.from_numpy(st[k]))
        adam.step = step - 1
        before = [a.copy() for a in go.arrays()]
        ad = new_adam_state(go, LR_INIT, step)
        ad["m1"], ad["m2"] = m1, m2
        loss_o = oracle.train_step(go, cam, BACKGROUND, tgt.cpu().numpy(), ad, st, degrees_to_use=0)
        loss = ctx.train_step(p, adam, cam, BACKGROUND, tgt, stats, degrees_to_use=0, sync_loss=True)
        what = f"step {step}"
        _check_frame(ctx, oracle, ctx.frame("out_img").cpu().numpy(), oracle.frame("out_img"), what)
        assert abs(loss - loss_o) <= 1e-6 * abs(loss_o), (what, loss, loss_o)
        for key in GRAD_KEYS:
            got, ref = ctx.frame(key).cpu().numpy(), oracle.frame(key)
            if key == "v_quat":
                # kNN initialisation makes every Gaussian isotropic (one scale for all
                # three axes), where the covariance does not depend on the rotation: the
                # true quaternion gradient is zero and both sides return the rounding
                # residue of terms the size of the scale gradient. That residue is
                # bounded against the scale gradient instead of compared relatively.
                d = float(np.linalg.norm(got.astype(np.float64) - ref))
                bound = GRAD_RTOL_L2 * float(np.linalg.norm(oracle.frame("v_scale").astype(np.float64)))
                assert d <= bound, (what, key, d, bound)
                continue
            r = rel_l2(got, ref)
            assert r <= GRAD_RTOL_L2, (what, key, r)
        # moments and updates of every group but the quaternions (group 2), whose
        # gradient is the rounding residue above: Adam turns a residue of either sign
        # into a full-size step (m1 / sqrt(m2)), on both sides alike
        for name, mg, mo in (("m1", adam.exp_avg, m1), ("m2", adam.exp_avg_sq, m2)):
            for gi, (a, b) in enumerate(zip(mg, mo)):
                if gi != 2:
                    assert rel_l2(a.cpu().numpy(), b) <= GRAD_RTOL_L2, (what, name, gi)
        if step > 1:  # step 1 moves every element by about +-lr whatever its gradient
            for gi, (b0, a, r) in enumerate(zip(before, p.numpy(), go.arrays())):
                if gi != 2:
                    assert rel_l2(a - b0, r - b0) <= GRAD_RTOL_L2, (what, "update", gi)
    for t, k in zip(stats, ("vis", "gn", "ms")):
        assert rel_l2(t.cpu().numpy(), st[k]) <= GRAD_RTOL_L2, k

    # densify with the statistics of the three steps, the street config's thresholds
    cap = 4 * n
    strides = [3, 3, 4, 3, 45, 1]
    bufs = [np.pad(a.reshape(n, s), ((0, cap - n), (0, 0))).astype(np.float32) for a, s in zip(go.arrays(), strides)]
    o1 = [np.pad(a.reshape(n, s), ((0, cap - n), (0, 0))).astype(np.float32) for a, s in zip(m1, strides)]
    o2 = [np.pad(a.reshape(n, s), ((0, cap - n), (0, 0))).astype(np.float32) for a, s in zip(m2, strides)]
    tb = [torch.from_numpy(b).cuda() for b in bufs]
    t1 = [torch.from_numpy(b).cuda() for b in o1]
    t2 = [torch.from_numpy(b).cuda() for b in o2]
    gstat = [torch.from_numpy(st[k]).cuda() for k in ("gn", "vis", "ms")]
    half_max_dim, seed = 512.0, (500 * 2654435761) & 0xFFFFFFFF
    kw = dict(grad_thresh=2e-4, size_thresh=0.01, screen_thresh=0.05, check_screen=1, cull_alpha=0.005,
              cull_scale=0.5, cull_screen=0.15, check_huge=0)
    new_o = oracle.densify(n, cap, bufs, o1, o2, st, half_max_dim, seed, **kw)
    new_n = ctx.densify(n, tb, t1, t2, gstat[0], gstat[1], gstat[2], half_max_dim, seed,
                        **{k: (bool(v) if k.startswith("check") else v) for k, v in kw.items()})
    assert new_n == new_o
    for gi in range(6):
        np.testing.assert_allclose(tb[gi].cpu().numpy()[:new_n], bufs[gi][:new_n], rtol=1e-6, atol=1e-7,
                                   err_msg=str(gi))
        assert np.array_equal(t1[gi].cpu().numpy()[:new_n], o1[gi][:new_n]), gi
        assert np.array_equal(t2[gi].cpu().numpy()[:new_n], o2[gi][:new_n]), gi


def test_serving_distribution_1080p_render(oracle):
    """1.5 M Gaussians of the serving distribution, a camera on the 5 m sphere, 1920 x 1080."""
    g = scenes.random_gaussians(1_500_000, 77)
    cam = scenes.sphere_camera(np.random.default_rng(78), 1920, 1080)
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context()
    img = ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND).cpu().numpy()
    _check_frame(ctx, oracle, img, img_o, "1080p")
    assert int(ctx.num_isects()) > 10_000_000
