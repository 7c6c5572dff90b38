"""Prior-guided extras on the GPU vs the CPU oracle (core/metal/bindings.h:43-77):
aux rasterization (expected depth, per-pixel background), the learned sky, the depth /
sky / fill prior losses, the affine exposure and the needle cap.

Bar: as the plain path -- images max-abs <= 1e-5, gradients relative L2 <= 1e-4,
integer data bit-exact. The transmittance and the expected-depth numerator carry the
plain path's few-ulp differences (exp evaluated in double on the device, glibc's
expf on the host) and are compared like images. The sky direction uses asin / atan2
and the depth residual log; the oracle calls the host's float functions, the kernels
evaluate them in double and round once, which differs in the last place for a small
share of inputs, so sky colours, sky gradients and depth-prior gradients are compared
within tolerance. The exposure-gradient sum runs in double in both, in another
order, so the exposure parameters after Adam are compared to a few ulps.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import scenes
from msplat_street_b200._lib import lib
from msplat_street_b200.backend import AdamState, Context, GaussianParams, PriorStep, ptr
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle, new_adam_state, set_prior
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, IMAGE_ATOL, max_abs, rel_l2
from prior_util import ALL, copy_prior, make_prior, restep

pytestmark = pytest.mark.gpu

GRAD_KEYS = ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")
MODES = [("aux",), ("aux", "sky"), ("aux", "depth"), ("exposure",), ("needle",), ALL]


@pytest.fixture(scope="module")
def oracle():
    o = Oracle("restatement")
    yield o
    set_prior(o, None)


def to_gpu(pr: dict) -> PriorStep:
    """The PriorStep of a prior_util dict, over CUDA copies of its arrays."""
    kw = {}
    for k, v in pr.items():
        if isinstance(v, np.ndarray):
            if k == "sky_frame":
                kw[k] = tuple(float(x) for x in v)
            else:
                kw[k] = torch.from_numpy(v.copy()).cuda()
        elif k not in ("sky_w", "sky_h", "prior_w", "prior_h"):
            kw[k] = v
    for k in ("aux", "sky", "exposure", "has_depth", "has_sky_mask", "mask_photometric"):
        if k in kw:
            kw[k] = bool(kw[k])
    return PriorStep(**kw)


def _camera():
    return prepare_cam(look_at((0.5, 0.4, 2.8), (0, 0, 0)), 150, 110, 170.0, 160.0, 74.0, 56.0)


def _scene():
    return scenes.random_gaussians(3000, 50, sh_degree=2)


@pytest.mark.parametrize("sky", [False, True], ids=["const_bg", "sky"])
def test_render_aux(oracle, sky):
    g, cam = _scene(), _camera()
    pr = make_prior(cam.width, cam.height, 8, ("aux", "sky") if sky else ("aux",))
    set_prior(oracle, pr)
    img_o = oracle.render(g, cam, BACKGROUND)
    ctx = Context()
    ctx.set_prior(to_gpu(pr))
    img = ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND).cpu().numpy()
    depth, final_t = (t.cpu().numpy() for t in ctx.render_aux_outputs())
    assert max_abs(final_t, oracle.frame("final_Ts")) <= IMAGE_ATOL
    np.testing.assert_allclose(depth, oracle.frame("out_depth"), rtol=1e-5, atol=1e-6)
    assert np.abs(depth).max() > 0.5  # Gaussians in front of the camera
    bg = ctx.frame("bg_img").cpu().numpy()
    assert max_abs(img, img_o) <= IMAGE_ATOL
    if sky:
        assert max_abs(bg, oracle.frame("bg_img")) <= IMAGE_ATOL
        assert np.abs(bg - np.tile(BACKGROUND, cam.width * cam.height)).max() > 0.1  # the sky is what shows
    else:
        assert np.array_equal(bg, np.tile(BACKGROUND, cam.width * cam.height))
    set_prior(oracle, None)
    ctx.set_prior(None)
    ctx.render(GaussianParams.from_numpy(g), cam, BACKGROUND)
    with pytest.raises(ValueError):
        ctx.render_aux_outputs()


@pytest.mark.parametrize("modes", MODES, ids=lambda m: "+".join(m))
def test_train_step_with_prior(oracle, modes):
    g, cam = _scene(), _camera()
    set_prior(oracle, None)
    gt = oracle.render(scenes.random_gaussians(3000, 51, sh_degree=2), cam, BACKGROUND)
    pr = make_prior(cam.width, cam.height, 8, modes)
    po = copy_prior(pr)
    set_prior(oracle, po)
    go = g.copy()
    ad = new_adam_state(go, C1_LRS, 1)
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss_o = oracle.train_step(go, cam, BACKGROUND, gt, ad, st)

    ctx = Context(keep_grads=True)
    ps = to_gpu(pr)
    ctx.set_prior(ps)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    loss = ctx.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, sync_loss=True)
    assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o)), (loss, loss_o)

    aux = "aux" in modes
    if aux:
        np.testing.assert_allclose(ctx.frame("out_depth").cpu().numpy(), oracle.frame("out_depth"), rtol=1e-5,
                                   atol=1e-6)
        va, va_o = ctx.frame("v_aux").cpu().numpy(), oracle.frame("v_aux")
        assert rel_l2(va, va_o) <= GRAD_RTOL_L2
        assert rel_l2(ctx.frame("v_depth").cpu().numpy(), oracle.frame("v_depth")) <= GRAD_RTOL_L2
        terms = ps.loss_terms.cpu().numpy()
        np.testing.assert_allclose(terms, po["loss_terms"], rtol=1e-5, atol=1e-12)
    if "exposure" in modes:
        assert max_abs(ctx.frame("out_adj").cpu().numpy(), oracle.frame("out_adj")) <= IMAGE_ATOL
        assert rel_l2(ctx.frame("v_adj").cpu().numpy(), oracle.frame("v_adj")) <= 1e-5
        np.testing.assert_allclose(ps.expo_params.cpu().numpy(), po["expo_params"], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(ps.expo_exp_avg.cpu().numpy(), po["expo_exp_avg"], rtol=1e-5, atol=1e-9)
        assert np.array_equal(ps.expo_grad.cpu().numpy(), np.zeros(12, np.float32))
    if "sky" in modes:
        assert rel_l2(ps.sky_grad.cpu().numpy(), po["sky_grad"]) <= GRAD_RTOL_L2
        assert max_abs(ps.sky_tex.cpu().numpy(), po["sky_tex"]) <= 1e-5
    assert rel_l2(ctx.frame("v_rendered").cpu().numpy(), oracle.frame("v_rendered")) <= 1e-5
    for key in GRAD_KEYS:
        got, ref = ctx.frame(key).cpu().numpy(), oracle.frame(key)
        assert rel_l2(got, ref) <= GRAD_RTOL_L2, (key, rel_l2(got, ref))
    for before, gpu, ref, nm in zip(g.arrays(), p.numpy(), go.arrays(),
                                    ("means", "scales", "quats", "dc", "rest", "opacities")):
        assert rel_l2(gpu - before, ref - before) <= 1e-3, nm
    if "needle" in modes:
        ls = p.numpy()[1].reshape(-1, 3)
        assert (ls.max(1) - np.median(ls, 1)).max() <= pr["log_max_scale_ratio"] + 1e-5
        assert np.array_equal(np.sort(ls, 1)[:, 2] - np.sort(ls, 1)[:, 1] <= pr["log_max_scale_ratio"] + 1e-5,
                              np.ones(g.n, bool))
    set_prior(oracle, None)


def test_prior_steps_track_the_oracle(oracle):
    """Five steps with every extra on, each started from the oracle's state, so the
    comparison stays per step; the prior arrays are carried by each side."""
    g, cam = _scene(), _camera()
    set_prior(oracle, None)
    gt = oracle.render(scenes.random_gaussians(3000, 51, sh_degree=2), cam, BACKGROUND)
    pr = make_prior(cam.width, cam.height, 8, ALL)
    go = g.copy()
    m1 = [np.zeros_like(a) for a in g.arrays()]
    m2 = [np.zeros_like(a) for a in g.arrays()]
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    ctx = Context(keep_grads=True)
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    stats = tuple(torch.zeros(g.n, device="cuda") for _ in range(3))
    for step in range(1, 6):
        restep(pr, step)
        ps = to_gpu(pr)  # this step's inputs, copied from the oracle's state
        for t, a in zip(p.tensors(), go.arrays()):
            t.copy_(torch.from_numpy(a))
        for t, a in zip(adam.exp_avg, m1):
            t.copy_(torch.from_numpy(a))
        for t, a in zip(adam.exp_avg_sq, m2):
            t.copy_(torch.from_numpy(a))
        adam.step = step - 1
        ctx.set_prior(ps)
        loss = ctx.train_step(p, adam, cam, BACKGROUND, torch.from_numpy(gt).cuda(), stats, sync_loss=True)
        set_prior(oracle, pr)
        ad = new_adam_state(go, C1_LRS, step)
        ad["m1"], ad["m2"] = m1, m2
        loss_o = oracle.train_step(go, cam, BACKGROUND, gt, ad, st)
        assert abs(loss - loss_o) <= 1e-6 * max(1.0, abs(loss_o)), (step, loss, loss_o)
        for key in GRAD_KEYS:
            assert rel_l2(ctx.frame(key).cpu().numpy(), oracle.frame(key)) <= GRAD_RTOL_L2, (step, key)
        assert rel_l2(ps.sky_grad.cpu().numpy(), pr["sky_grad"]) <= GRAD_RTOL_L2, step
        np.testing.assert_allclose(ps.expo_params.cpu().numpy(), pr["expo_params"], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(ps.loss_terms.cpu().numpy(), pr["loss_terms"], rtol=1e-5, atol=1e-12)
    set_prior(oracle, None)


def test_set_prior_rejects_inconsistent_fields():
    ctx = Context()
    with pytest.raises(ValueError):
        ctx.set_prior(PriorStep(aux=True, sky=True))  # sky without its texture
    tex = torch.zeros((4, 8, 3), device="cuda")
    with pytest.raises(ValueError):
        ctx.set_prior(PriorStep(aux=True, sky=True, sky_tex=tex, sky_grad=torch.zeros_like(tex)))  # no moments
    with pytest.raises(ValueError):
        ctx.set_prior(PriorStep(exposure=True, expo_params=torch.zeros((2, 12), device="cuda")))
    with pytest.raises(ValueError):
        ctx.set_prior(PriorStep(prior_aux=torch.zeros((4, 4, 4), device="cuda")))  # wrong dtype
    e = torch.zeros((2, 12), device="cuda")
    with pytest.raises(ValueError):  # a camera without an exposure row
        ctx.set_prior(PriorStep(exposure=True, expo_params=e, expo_exp_avg=e.clone(), expo_exp_avg_sq=e.clone(),
                                cam_index=2))
    aux = torch.zeros(4 * 4 * 4 + 1, dtype=torch.uint8, device="cuda")[1:].view(4, 4, 4)
    with pytest.raises(ValueError):  # not 4-byte aligned
        ctx.set_prior(PriorStep(aux=True, prior_aux=aux))
    ctx.set_prior(None)


def test_render_backward_refuses_aux_frames():
    g, cam = _scene(), _camera()
    ctx = Context()
    p = GaussianParams.from_numpy(g)
    ctx.set_prior(PriorStep(aux=True))
    ctx.render(p, cam, BACKGROUND)
    v = torch.ones((cam.height, cam.width, 3), device="cuda")
    grads = [torch.zeros_like(t) for t in p.tensors()]
    bg = np.asarray(BACKGROUND, np.float32)
    status = lib().msplat_cuda_render_backward(
        ctx.handle, p.n, ptr(p.means), ptr(p.scales), 1.0, ptr(p.quats), cam.viewmat.ctypes.data,
        cam.projmat.ctypes.data, cam.fx, cam.fy, cam.cx, cam.cy, cam.height, cam.width, cam.tiles_x, cam.tiles_y,
        0.01, p.sh_degree, p.sh_degree, cam.cam_pos.ctypes.data, bg.ctypes.data, ptr(v), *[ptr(t) for t in grads])
    assert status == 5  # MSPLAT_CUDA_EUNSUPPORTED


def test_batch_entry_points_refuse_a_prior():
    g, cam = _scene(), _camera()
    ctx = Context()
    p = GaussianParams.from_numpy(g)
    ctx.set_prior(PriorStep(aux=True))
    from msplat_street_b200.backend import BatchItem
    with pytest.raises(NotImplementedError):
        ctx.render_batch([BatchItem(p, cam, BACKGROUND)])
    ctx.set_prior(None)
    assert len(ctx.render_batch([BatchItem(p, cam, BACKGROUND)])) == 1


@pytest.mark.parametrize("shape", [1, 2], ids=["16x8", "8x8"])
def test_block_shapes_with_prior_and_stored_transmittance(shape):
    """The forward's block shapes (raster_shape) in the aux rasterizer (a prior with the
    sky, the depth prior and the exposure) and with stored transmittance: the same
    render, aux outputs, loss and updated parameters, bit for bit, as whole-tile blocks."""
    g, cam = _scene(), _camera()
    results = []
    for s in (0, shape):
        out = []
        # aux render and training step with the full prior
        ctx = Context()
        ctx.set_raster_shape(s)
        pr = to_gpu(make_prior(cam.width, cam.height, 8, ALL))
        ctx.set_prior(pr)
        p = GaussianParams.from_numpy(g)
        out.append(ctx.render(p, cam, BACKGROUND).clone())
        out.extend(t.clone() for t in ctx.render_aux_outputs())
        tgt = out[0].clone()
        adam = AdamState.zeros_like(p, C1_LRS)
        st = tuple(torch.zeros(p.n, device="cuda") for _ in range(3))
        out.append(torch.tensor([ctx.train_step(p, adam, cam, BACKGROUND, tgt.flip(0).contiguous(), st,
                                                sync_loss=True)]))
        out.extend(t.clone() for t in p.tensors())
        ctx.set_prior(None)
        # plain step with stored transmittance
        ctx2 = Context(store_transmittance=16)
        ctx2.set_raster_shape(s)
        q = GaussianParams.from_numpy(g)
        adam2 = AdamState.zeros_like(q, C1_LRS)
        st2 = tuple(torch.zeros(q.n, device="cuda") for _ in range(3))
        out.append(torch.tensor([ctx2.train_step(q, adam2, cam, BACKGROUND, tgt.flip(0).contiguous(), st2,
                                                 sync_loss=True)]))
        out.extend(t.clone() for t in q.tensors())
        out.append(ctx2.frame("final_idx").clone())
        results.append([t.cpu() for t in out])
    for a, b in zip(*results):
        assert torch.equal(a, b)
