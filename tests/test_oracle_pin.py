"""Pins the oracle restatement (oracle/msplat_oracle.cpp) to the reference (no GPU).

Two anchors:
 * golden vectors in tests/golden/*.npz, produced by the reference's own CPU backend
   (tests/golden/make_golden.py) -- always checked;
 * the reference backend itself, compiled from its sources into oracle/_ref -- checked
   on larger seeded cases when that build is present.
The restatement must reproduce the reference bit for bit.
"""
import os

import numpy as np
import pytest

from msplat_street_b200 import scenes
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle, available, new_adam_state, set_prior
from parity_util import BACKGROUND, C1_LRS
from prior_util import ALL, copy_prior, make_prior, restep

PRIOR_ARRAYS = ("sky_tex", "sky_exp_avg", "sky_exp_avg_sq", "sky_grad", "loss_terms", "expo_params",
                "expo_exp_avg", "expo_exp_avg_sq", "expo_grad")
PRIOR_FRAMES = ("out_depth", "bg_img", "final_Ts", "v_aux", "v_depth", "out_adj", "v_adj")
GRADS = ("v_rendered", "v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def rest():
    return Oracle("restatement")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


# ---- golden vectors -------------------------------------------------------------

def _golden_scene(seed):
    return scenes.random_gaussians(400, seed, log_scale_mean=-3.0)


def _golden_camera():
    return prepare_cam(look_at((0.3, -0.2, 2.6), (0.0, 0.1, 0.0)), 70, 46, 80.0, 76.0, 35.4, 22.8)


def test_golden_render(rest):
    gv = _load("render_train.npz")
    g = _golden_scene(10)
    cam = _golden_camera()
    img = rest.render(g, cam, BACKGROUND)
    assert np.array_equal(img, gv["image"])
    radii = rest.frame("radii")
    assert np.array_equal(radii, gv["render_radii"])
    vis = radii > 0
    for k in ("tile_start", "tile_end", "isect_gid", "final_idx", "final_Ts"):
        assert np.array_equal(rest.frame(k), gv["render_" + k]), k
    for k, w in (("xys", 2), ("depths", 1), ("conics", 3), ("colors", 3)):
        assert np.array_equal(rest.frame(k).reshape(-1, w)[vis], gv["render_" + k].reshape(-1, w)[vis]), k


def test_golden_train_steps(rest):
    gv = _load("render_train.npz")
    g = _golden_scene(10)
    cam = _golden_camera()
    gt = gv["gt"]
    m1 = [np.zeros_like(a) for a in g.arrays()]
    m2 = [np.zeros_like(a) for a in g.arrays()]
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    for step in (1, 2):
        ad = new_adam_state(g, C1_LRS, step)
        ad["m1"], ad["m2"] = m1, m2
        loss = rest.train_step(g, cam, BACKGROUND, gt, ad, st)
        assert np.float32(loss) == gv[f"step{step}_loss"]
        for k in ("v_rendered", "v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat"):
            assert np.array_equal(rest.frame(k), gv[f"step{step}_{k}"]), (step, k)
        for name, a in zip(("means", "scales", "quats", "dc", "rest", "opac"), g.arrays()):
            assert np.array_equal(a, gv[f"step{step}_param_{name}"]), (step, name)
    for k in ("vis", "gn", "ms"):
        assert np.array_equal(st[k], gv["stats_" + k]), k


def test_golden_densify(rest):
    gv = _load("densify.npz")
    n, cap = 300, 1000
    bufs = [gv[f"in_{i}"].copy() for i in range(6)]
    m1 = [gv[f"in_m1_{i}"].copy() for i in range(6)]
    m2 = [gv[f"in_m2_{i}"].copy() for i in range(6)]
    stats = {k: gv["in_" + k] for k in ("vis", "gn", "ms")}
    new_n = rest.densify(n, cap, bufs, m1, m2, stats, half_max_dim=40.0, seed=12345)
    assert new_n == int(gv["new_n"])
    for i in range(6):
        assert np.array_equal(bufs[i][:new_n], gv[f"out_{i}"]), i
        assert np.array_equal(m1[i][:new_n], gv[f"out_m1_{i}"]), i
        assert np.array_equal(m2[i][:new_n], gv[f"out_m2_{i}"]), i


def test_golden_primitives(rest):
    gv = _load("primitives.npz")
    sort_cases = sorted({k.rsplit("_", 1)[0] for k in gv if k.startswith("sort_")})
    assert len(sort_cases) == 7
    for case in sort_cases:
        bits = int(case.split("_")[2])
        k, v = rest.radix_sort(gv[case + "_keys"], bits)
        assert np.array_equal(k, gv[case + "_sorted"]), case
        assert np.array_equal(v, gv[case + "_order"]), case
        ref = np.argsort(gv[case + "_keys"] & np.uint64((1 << bits) - 1 if bits < 64 else 2 ** 64 - 1),
                         kind="stable")
        assert np.array_equal(v, ref), case  # stable, as numpy's stable argsort
    md = rest.knn3_mean_dist(gv["knn_points"])
    assert np.array_equal(md, gv["knn_mean_dist"])
    s, q, d, o = rest.init_gaussians(gv["knn_points"], gv["init_rgb"], 42, float(np.log(0.1 / 0.9)))
    for a, b in ((s, "init_scales"), (q, "init_quats"), (d, "init_dc"), (o, "init_opac")):
        assert np.array_equal(a, gv[b]), b


def test_knn_matches_bruteforce(rest):
    """The reference's kNN test clouds (tests/test_msplat.py:444-465), against float64
    brute force."""
    rng = np.random.default_rng(7)
    clouds = {
        "uniform": rng.uniform(-1, 1, (3000, 3)),
        "street": np.vstack([np.c_[rng.uniform(-20, 20, 2000), rng.normal(0, 0.02, 2000), rng.uniform(0, 80, 2000)],
                             np.c_[8 + rng.normal(0, 0.05, 800), rng.uniform(0, 10, 800), rng.uniform(0, 80, 800)],
                             rng.normal(0, 300, (200, 3))]),
        "duplicates": np.vstack([rng.uniform(-1, 1, (500, 3)), np.repeat(rng.uniform(-1, 1, (8, 3)), 4, axis=0)]),
    }
    for name, pts in clouds.items():
        pts = pts.astype(np.float32)
        d2 = ((pts[:, None, :].astype(np.float64) - pts[None, :, :]) ** 2).sum(-1)
        np.fill_diagonal(d2, np.inf)
        want = np.sqrt(np.sort(d2, axis=1)[:, :3]).mean(axis=1)
        np.testing.assert_allclose(rest.knn3_mean_dist(pts), want, rtol=1e-4, atol=1e-6, err_msg=name)


def test_golden_prior_steps(rest):
    """Learned sky, depth / sky / fill priors, exposure and needle cap together
    (core/cpu/msplat_cpu.cpp:787-964, 1204-1327)."""
    gv = _load("prior.npz")
    g = _golden_scene(10)
    cam = _golden_camera()
    pr = make_prior(70, 46, 3, ALL)
    try:
        set_prior(rest, pr)
        assert np.array_equal(rest.render(g, cam, BACKGROUND), gv["image"])
        for k in ("out_depth", "bg_img", "final_Ts"):
            assert np.array_equal(rest.frame(k), gv["render_" + k]), k
        m1 = [np.zeros_like(a) for a in g.arrays()]
        m2 = [np.zeros_like(a) for a in g.arrays()]
        st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
        for step in (1, 2):
            set_prior(rest, restep(pr, step))
            ad = new_adam_state(g, C1_LRS, step)
            ad["m1"], ad["m2"] = m1, m2
            assert np.float32(rest.train_step(g, cam, BACKGROUND, gv["gt"], ad, st)) == gv[f"step{step}_loss"]
            for k in GRADS + PRIOR_FRAMES:
                assert np.array_equal(rest.frame(k), gv[f"step{step}_{k}"]), (step, k)
            for name, a in zip(("means", "scales", "quats", "dc", "rest", "opac"), g.arrays()):
                assert np.array_equal(a, gv[f"step{step}_param_{name}"]), (step, name)
            for k in PRIOR_ARRAYS:
                assert np.array_equal(pr[k], gv[f"step{step}_prior_{k}"]), (step, k)
        # the extras were exercised: sky seen, priors and exposure moved, needles capped
        assert gv["step1_prior_loss_terms"][:3].min() > 0
        assert not np.array_equal(gv["step2_prior_sky_tex"], make_prior(70, 46, 3, ALL)["sky_tex"])
        ls = gv["step2_param_scales"]
        spread = ls.max(1) - np.median(ls, 1)
        assert spread.max() <= 0.7 + 1e-6
    finally:
        set_prior(rest, None)


# ---- against the reference build itself (where it was compiled) ------------------

needs_ref = pytest.mark.skipif(not available("reference"), reason="reference CPU backend not built here")


@needs_ref
@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_reference_render_and_steps(rest, deg):
    ref = Oracle("reference")
    g = scenes.random_gaussians(4000, 30 + deg, sh_degree=deg)
    cam = prepare_cam(look_at((0.5, 0.4, 2.8), (0, 0, 0)), 150, 110, 170.0, 160.0, 74.0, 56.0)
    assert np.array_equal(rest.render(g, cam, BACKGROUND), ref.render(g, cam, BACKGROUND))
    for k in ("radii", "tile_start", "tile_end", "isect_gid", "final_idx"):
        assert np.array_equal(rest.frame(k), ref.frame(k)), k
    gt = ref.render(scenes.random_gaussians(4000, 99, sh_degree=deg), cam, BACKGROUND)
    ga, gb = g.copy(), g.copy()
    sa = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    sb = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    ma = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
    mb = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
    for step in (1, 2, 3):
        aa = new_adam_state(ga, C1_LRS, step)
        aa["m1"], aa["m2"] = ma
        ab = new_adam_state(gb, C1_LRS, step)
        ab["m1"], ab["m2"] = mb
        la = rest.train_step(ga, cam, BACKGROUND, gt, aa, sa, degrees_to_use=min(step - 1, deg))
        lb = ref.train_step(gb, cam, BACKGROUND, gt, ab, sb, degrees_to_use=min(step - 1, deg))
        assert la == lb
        for k in ("v_rendered", "v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat"):
            assert np.array_equal(rest.frame(k), ref.frame(k)), (step, k)
        for a, b in zip(ga.arrays(), gb.arrays()):
            assert np.array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("modes", [("aux",), ("aux", "sky"), ("aux", "depth"), ("exposure",), ("needle",), ALL],
                         ids=lambda m: "+".join(m))
def test_reference_prior_steps(rest, modes):
    """Each prior-guided extra alone and all together, against the reference, on a
    150x110 view: render frames, three training steps, every updated array."""
    ref = Oracle("reference")
    cam = prepare_cam(look_at((0.5, 0.4, 2.8), (0, 0, 0)), 150, 110, 170.0, 160.0, 74.0, 56.0)
    g = scenes.random_gaussians(3000, 50, sh_degree=2)
    set_prior(ref, None)
    gt = ref.render(scenes.random_gaussians(3000, 51, sh_degree=2), cam, BACKGROUND)
    pr = make_prior(150, 110, 8, modes)
    pa, pb = copy_prior(pr), copy_prior(pr)
    try:
        set_prior(rest, pa)
        set_prior(ref, pb)
        assert np.array_equal(rest.render(g, cam, BACKGROUND), ref.render(g, cam, BACKGROUND))
        for k in ("out_depth", "bg_img", "final_Ts"):
            assert np.array_equal(rest.frame(k), ref.frame(k)), k
        ga, gb = g.copy(), g.copy()
        ma = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
        mb = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
        sa = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
        sb = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
        for step in (1, 2, 3):
            set_prior(rest, restep(pa, step))
            set_prior(ref, restep(pb, step))
            aa = new_adam_state(ga, C1_LRS, step)
            aa["m1"], aa["m2"] = ma
            ab = new_adam_state(gb, C1_LRS, step)
            ab["m1"], ab["m2"] = mb
            assert rest.train_step(ga, cam, BACKGROUND, gt, aa, sa) == ref.train_step(gb, cam, BACKGROUND, gt, ab, sb)
            # frames a mode does not write keep whatever an earlier call left there
            frames = [k for k in PRIOR_FRAMES if ("aux" in modes or k in ("final_Ts", "v_depth"))
                      and ("exposure" in modes or k not in ("out_adj", "v_adj"))]
            for k in GRADS + tuple(frames):
                assert np.array_equal(rest.frame(k), ref.frame(k)), (step, k)
            for a, b in zip(ga.arrays(), gb.arrays()):
                assert np.array_equal(a, b)
            for k in PRIOR_ARRAYS:
                if k in pa:
                    assert np.array_equal(pa[k], pb[k]), (step, k)
    finally:
        set_prior(rest, None)
        set_prior(ref, None)


@needs_ref
def test_reference_small_config(rest):
    """The 10k-Gaussian 256x256 plain config: render and three training steps."""
    ref = Oracle("reference")
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    assert np.array_equal(rest.render(g, cam, BACKGROUND), ref.render(g, cam, BACKGROUND))
    gt = ref.render(scenes.small_scene(1), cam, BACKGROUND)
    ga, gb = g.copy(), g.copy()
    ma = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
    mb = [[np.zeros_like(a) for a in g.arrays()] for _ in range(2)]
    sa = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    sb = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    for step in (1, 2, 3):
        aa = new_adam_state(ga, C1_LRS, step)
        aa["m1"], aa["m2"] = ma
        ab = new_adam_state(gb, C1_LRS, step)
        ab["m1"], ab["m2"] = mb
        assert rest.train_step(ga, cam, BACKGROUND, gt, aa, sa) == ref.train_step(gb, cam, BACKGROUND, gt, ab, sb)
        for a, b in zip(ga.arrays(), gb.arrays()):
            assert np.array_equal(a, b)


@needs_ref
def test_reference_densify_and_reset(rest):
    ref = Oracle("reference")
    rng = np.random.default_rng(5)
    n, cap = 2000, 6000
    g = scenes.random_gaussians(n, 40, log_scale_mean=-4.0, log_scale_std=1.5)
    strides = [3, 3, 4, 3, 45, 1]
    mk = lambda: [np.pad(a.reshape(n, s), ((0, cap - n), (0, 0))).astype(np.float32)  # noqa: E731
                  for a, s in zip(g.arrays(), strides)]
    ba, bb = mk(), mk()
    m = [(rng.random((cap, s)).astype(np.float32), rng.random((cap, s)).astype(np.float32)) for s in strides]
    m1a, m2a = [x[0].copy() for x in m], [x[1].copy() for x in m]
    m1b, m2b = [x[0].copy() for x in m], [x[1].copy() for x in m]
    stats = {"vis": rng.integers(0, 4, n).astype(np.float32), "gn": (rng.random(n) * 2e-3).astype(np.float32),
             "ms": (rng.random(n) * 0.3).astype(np.float32)}
    for check_screen, check_huge in ((1, 1), (0, 1), (1, 0)):
        na = rest.densify(n, cap, [b.copy() for b in ba], [x.copy() for x in m1a], [x.copy() for x in m2a], stats,
                          60.0, 777, check_screen=check_screen, check_huge=check_huge)
        nb = ref.densify(n, cap, [b.copy() for b in bb], [x.copy() for x in m1b], [x.copy() for x in m2b], stats,
                         60.0, 777, check_screen=check_screen, check_huge=check_huge)
        assert na == nb
    na = rest.densify(n, cap, ba, m1a, m2a, stats, 60.0, 777)
    nb = ref.densify(n, cap, bb, m1b, m2b, stats, 60.0, 777)
    assert na == nb
    for x, y in zip(ba + m1a + m2a, bb + m1b + m2b):
        assert np.array_equal(x[:na], y[:nb])
    oa, ob = ba[5][:na, 0].copy(), bb[5][:nb, 0].copy()
    rest.opacity_reset(oa, m1a[5][:na, 0].copy(), m2a[5][:na, 0].copy(), na, -1.3862943611198906)
    ref.opacity_reset(ob, m1b[5][:nb, 0].copy(), m2b[5][:nb, 0].copy(), nb, -1.3862943611198906)
    assert np.array_equal(oa, ob)


@needs_ref
def test_reference_image_ops(rest):
    ref = Oracle("reference")
    rng = np.random.default_rng(3)
    a = rng.random((37, 53, 3)).astype(np.float32)
    b = np.clip(a + rng.normal(0, 0.05, a.shape), 0, 1).astype(np.float32)
    assert np.array_equal(rest.image_metrics(a, b), ref.image_metrics(a, b))
    assert np.array_equal(rest.resize_area(a, 20, 14), ref.resize_area(a, 20, 14))
    u8 = rng.integers(0, 256, (37, 53, 4)).astype(np.uint8)
    assert np.array_equal(rest.resize_area(u8, 53, 37), ref.resize_area(u8, 53, 37))
    assert np.array_equal(rest.resize_area(u8, 17, 11), ref.resize_area(u8, 17, 11))
    assert np.array_equal(rest.pack_rgba8(a * 1.2 - 0.1), ref.pack_rgba8(a * 1.2 - 0.1))
    intr, dist = [48.0, 46.0, 26.2, 18.7], [-0.12, 0.03, 0.001, -0.002, 0.004]
    assert np.array_equal(rest.undistort(a, intr, dist, 2, 1, 49, 34), ref.undistort(a, intr, dist, 2, 1, 49, 34))
    t = rng.random(500).astype(np.float32)
    t[::7] = 1.0  # alpha 0 -> depth 0
    dn = rng.random(500).astype(np.float32) * 3
    for x, y in zip(rest.finalize_depth(dn, t, 0.5), ref.finalize_depth(dn, t, 0.5)):
        assert np.array_equal(x, y)


# ---- the oracle's gradients against float64 finite differences --------------------

@pytest.mark.parametrize("view_dependent", [False, True])
def test_oracle_gradients_match_finite_differences(rest, view_dependent):
    """Like the reference's own gradient check (tests/gradcheck.cpp), on the smooth
    64-Gaussian 32x32 scenes, against tests/golden/fd_smooth.npz."""
    from grad_util import fd_agreement, oracle_param_grads
    from smooth_scenes import smooth_scene
    g, cam, gt = smooth_scene(view_dependent=view_dependent)
    fx = _load("fd_smooth.npz")
    tag = "vd" if view_dependent else "flat"
    fd = [fx[f"{tag}_{k}"] for k in ("means", "scales", "quats", "dc", "rest", "opacities")]
    ad = new_adam_state(g, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    rest.train_step(g.copy(), cam, BACKGROUND, gt, ad, st)
    grads = oracle_param_grads(rest, g, cam, 3)
    bad, checked, cos = fd_agreement(grads, fd, skip=(0,) if view_dependent else ())
    assert bad == 0 and cos > 0.9999, (bad, checked, cos)
