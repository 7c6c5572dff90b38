"""The batched multi-view training step (msplat_cuda_train_batch) on the GPU.

Its contract: gradients summed over the views (each view's loss scaled as the
single-view step scales it), one Adam step, statistics advanced once per view; a
one-view batch is the single-view step. Checked here against the single-view step,
against the sum of the differentiable path's per-view gradients, against the oracle's
per-view gradients, and graph replay against eager execution.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import autograd as ag
from msplat_street_b200 import scenes
from msplat_street_b200.backend import AdamState, Context, GaussianParams
from msplat_street_b200.camera import look_at, prepare_cam
from oracle_lib import Oracle, new_adam_state
from parity_util import BACKGROUND, C1_LRS, GRAD_RTOL_L2, rel_l2

pytestmark = pytest.mark.gpu

SH_C0 = 0.28209479177387814


def _cams():
    """Three views of the small scene at different resolutions (one not a multiple of 16)."""
    return [
        scenes.small_camera(),
        prepare_cam(look_at((0.8, 0.3, 2.6), (0, 0, 0)), 200, 136, 180.0, 170.0, 97.5, 70.25),
        prepare_cam(look_at((-1.2, -0.4, 2.4), (0, 0, 0)), 320, 240, 260.0, 260.0, 160.0, 120.0),
    ]


def _targets(cams):
    o = Oracle()
    tgt = scenes.small_scene(1)
    return [torch.from_numpy(o.render(tgt, c, BACKGROUND)).cuda() for c in cams]


def _stats(n):
    return tuple(torch.zeros(n, device="cuda") for _ in range(3))


def test_one_view_batch_equals_train_step():
    g = scenes.small_scene(0)
    cam = scenes.small_camera()
    gt = _targets([cam])[0]
    p1, p2 = GaussianParams.from_numpy(g), GaussianParams.from_numpy(g)
    a1, a2 = AdamState.zeros_like(p1, C1_LRS), AdamState.zeros_like(p2, C1_LRS)
    s1, s2 = _stats(g.n), _stats(g.n)
    c1, c2 = Context(), Context()
    for _ in range(3):
        l1 = c1.train_step(p1, a1, cam, BACKGROUND, gt, s1, sync_loss=True)
        l2 = c2.train_batch(p2, a2, [(cam, gt)], BACKGROUND, s2)
        assert l1 == float(l2[0])
    for x, y in zip(p1.tensors() + a1.exp_avg + a1.exp_avg_sq + list(s1),
                    p2.tensors() + a2.exp_avg + a2.exp_avg_sq + list(s2)):
        assert torch.equal(x, y)


def _view_grads(p, cam, gt, dtu=None):
    q = GaussianParams(*[t.clone().requires_grad_(True) for t in p.tensors()])
    loss = ag.ssim_l1_loss(ag.render(q, cam, BACKGROUND, degrees_to_use=dtu), gt)
    loss.backward()
    return [t.grad for t in q.tensors()], float(loss.detach())


@pytest.mark.parametrize("dtu", [3, 1])
def test_batch_gradients_are_the_sum_of_view_gradients(dtu):
    g = scenes.small_scene(0)
    cams = _cams()
    gts = _targets(cams)
    p = GaussianParams.from_numpy(g)
    grads = [torch.empty_like(t) for t in p.tensors()]
    losses = Context().train_batch(p, None, list(zip(cams, gts)), BACKGROUND, grads=grads, degrees_to_use=dtu)
    ref = None
    for k, (c, t) in enumerate(zip(cams, gts)):
        gv, lv = _view_grads(p, c, t, dtu)
        assert abs(lv - float(losses[k])) <= 1e-6 * max(1.0, abs(lv))
        ref = gv if ref is None else [a + b for a, b in zip(ref, gv)]
    for nm, a, b in zip(("means", "scales", "quats", "dc", "rest", "opacities"), grads, ref):
        assert torch.allclose(a, b.reshape(a.shape), rtol=1e-6, atol=1e-12), (nm, float((a - b).abs().max()))


def test_batch_gradients_match_oracle():
    g = scenes.small_scene(0)
    cams = _cams()
    gts = _targets(cams)
    p = GaussianParams.from_numpy(g)
    grads = [torch.empty_like(t) for t in p.tensors()]
    Context().train_batch(p, None, list(zip(cams, gts)), BACKGROUND, grads=grads)
    o = Oracle()
    ref = {k: 0.0 for k in ("v_mean3d", "v_scale", "v_quat", "v_opacity", "v_rgb")}
    for c, t in zip(cams, gts):
        go = g.copy()
        ad = new_adam_state(go, C1_LRS, 1)
        st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
        o.train_step(go, c, BACKGROUND, t.cpu().numpy(), ad, st)
        for k in ref:
            ref[k] = ref[k] + o.frame(k).astype(np.float64)
    got = [x.cpu().numpy() for x in grads]
    assert rel_l2(got[0], ref["v_mean3d"].reshape(got[0].shape)) <= GRAD_RTOL_L2
    assert rel_l2(got[1], ref["v_scale"].reshape(got[1].shape)) <= GRAD_RTOL_L2
    assert rel_l2(got[2], ref["v_quat"].reshape(got[2].shape)) <= GRAD_RTOL_L2
    assert rel_l2(got[5].reshape(-1), ref["v_opacity"].reshape(-1)) <= GRAD_RTOL_L2
    assert rel_l2(got[3], SH_C0 * ref["v_rgb"].reshape(got[3].shape)) <= GRAD_RTOL_L2


def test_batch_adam_step_uses_summed_gradients():
    g = scenes.small_scene(0)
    cams = _cams()
    gts = _targets(cams)
    views = list(zip(cams, gts))
    p = GaussianParams.from_numpy(g)
    grads = [torch.empty_like(t) for t in p.tensors()]
    Context().train_batch(p, None, views, BACKGROUND, grads=grads)
    q = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(q, C1_LRS)
    st = _stats(g.n)
    Context().train_batch(q, adam, views, BACKGROUND, st)
    ss, bc2 = adam.step_scalars()
    b1, b2, eps = np.float32(0.9), np.float32(0.999), np.float32(1e-8)
    vis_any = st[0] > 0
    for k, (x0, xg, xq) in enumerate(zip(p.tensors(), grads, q.tensors())):
        gr = xg.double()
        m = (1 - 0.9) * gr
        v = (1 - 0.999) * gr * gr
        upd = float(ss[k]) * m / (torch.sqrt(v) / float(bc2[k]) + 1e-8)
        want = x0.double() - upd
        if k in (3, 4):  # SH groups: Adam only where some view sees the Gaussian
            want = torch.where(vis_any.reshape((-1,) + (1,) * (x0.dim() - 1)), want, x0.double())
        assert torch.allclose(xq.double(), want, rtol=0, atol=1e-6), k
    # statistics: one visit per view that sees the Gaussian
    per_view = [Context() for _ in cams]
    vis_sum = torch.zeros(g.n, device="cuda")
    for c, (cam, gt) in zip(per_view, views):
        s1 = _stats(g.n)
        c.train_step(GaussianParams.from_numpy(g), AdamState.zeros_like(q, C1_LRS), cam, BACKGROUND, gt, s1)
        vis_sum += s1[0]
    assert torch.equal(st[0], vis_sum)


def _street_views(seed=0, n_views=6):
    rng = np.random.default_rng(seed)
    res = [(64, 48), (96, 64), (128, 80), (160, 96)]
    out = []
    for k in range(n_views):
        w, h = res[int(rng.integers(len(res)))]
        eye = (float(rng.uniform(-0.5, 0.5)), float(rng.uniform(-0.3, 0.3)), float(rng.uniform(2.4, 3.2)))
        out.append(prepare_cam(look_at(eye, (0, 0, 0)), w, h, 0.9 * w, 0.9 * w, w / 2, h / 2))
    return out


def _run(ctx, g, batches, cams, gts):
    p = GaussianParams.from_numpy(g)
    adam = AdamState.zeros_like(p, C1_LRS)
    st = _stats(g.n)
    losses = []
    for b in batches:
        losses.append(ctx.train_batch(p, adam, [(cams[i], gts[i]) for i in b], BACKGROUND, st))
    torch.cuda.synchronize()
    return p, adam, st, losses


def test_graph_replay_equals_eager_steps():
    g = scenes.small_scene(0)
    cams = _street_views()
    gts = _targets(cams)
    rng = np.random.default_rng(3)
    batches = [list(rng.choice(len(cams), 3, replace=False)) for _ in range(8)]
    eager = _run(Context(), g, batches, cams, gts)
    cg = Context()
    cg.set_graph(True)
    graph = _run(cg, g, batches, cams, gts)
    for x, y in zip(eager[0].tensors() + eager[1].exp_avg + list(eager[2]),
                    graph[0].tensors() + graph[1].exp_avg + list(graph[2])):
        assert torch.equal(x, y)
    for a, b in zip(eager[3], graph[3]):
        assert np.array_equal(a, b)
    s = cg.graph_stats()
    assert s["replays"] >= 4 and s["captures"] >= 1


def test_graph_overflow_repeats_the_step():
    """A replay whose intersections exceed the capacity sized by earlier steps changes
    nothing and is repeated without the graph: Gaussians drawn 3x larger (glob_scale)
    cover about 9x the tiles."""
    g = scenes.small_scene(0)
    cam = scenes.small_camera(128, 128, 150.0)
    gt = _targets([cam])[0]
    scales = [1.0, 1.0, 1.0, 3.0, 3.0]
    res = []
    for graph in (False, True):
        ctx = Context()
        ctx.set_graph(graph)
        p = GaussianParams.from_numpy(g)
        adam = AdamState.zeros_like(p, C1_LRS)
        st = _stats(g.n)
        for gs in scales:
            ctx.train_batch(p, adam, [(cam, gt)], BACKGROUND, st, glob_scale=gs)
        torch.cuda.synchronize()
        res.append((p, st, ctx))
    for x, y in zip(res[0][0].tensors() + list(res[0][1]), res[1][0].tensors() + list(res[1][1])):
        assert torch.equal(x, y)
    stats = res[1][2].graph_stats()
    assert stats["overflows"] >= 1 and stats["replays"] >= 2
