"""Depth-chunked compositing in the oracle (core/metal/msplat_metal.metal:2641-3030)
against its one-pass compositing (core/cpu), on the CPU.

A tile whose list fits in one piece composites exactly as one pass (transmittance,
last contributor and gradients bit for bit; the image within one rounding of the
merge's fused background term). Long lists split into pieces differ from one pass by
what each piece's own early stop lets through: measured 3.5e-4 max-abs on the image
and about 1.2 % relative L2 on the gradients for the scene below."""
import numpy as np
import pytest

from msplat_street_b200 import scenes
from oracle_lib import Oracle, new_adam_state, set_option
from parity_util import BACKGROUND, C1_LRS, rel_l2

GRADS = ("v_xy", "v_conic", "v_rgb", "v_opacity", "v_mean3d", "v_scale", "v_quat")


@pytest.fixture()
def oracle():
    o = Oracle("restatement")
    yield o
    set_option(o, "chunk_size", 0)


def _step(o, g, cam, chunk):
    set_option(o, "chunk_size", chunk)
    gt = np.random.default_rng(1).random((cam.height, cam.width, 3)).astype(np.float32)
    go = g.copy()
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    loss = o.train_step(go, cam, BACKGROUND, gt, new_adam_state(go, C1_LRS, 1), st)
    keys = ("out_img", "final_Ts", "final_idx", "tile_start", "tile_end", "chunk_first") + GRADS
    return loss, {k: o.frame(k).copy() for k in keys}


def _long_lists():
    return scenes.random_gaussians(20000, 3, log_scale_mean=-2.0), scenes.small_camera(96, 64, 110.0)


def test_items_per_tile(oracle):
    g, cam = _long_lists()
    for chunk in (64, 512):
        _, f = _step(oracle, g, cam, chunk)
        lens = f["tile_end"] - f["tile_start"]
        assert lens.max() > 8 * chunk  # many pieces per tile
        want = np.concatenate([[0], np.cumsum((lens + chunk - 1) // chunk)])
        assert np.array_equal(f["chunk_first"], want)


def test_one_piece_is_one_pass(oracle):
    g, cam = scenes.random_gaussians(1500, 8), scenes.small_camera(80, 80, 100.0)
    loss0, a = _step(oracle, g, cam, 0)
    assert a["chunk_first"].size == 0
    lens = a["tile_end"] - a["tile_start"]
    loss1, b = _step(oracle, g, cam, int(lens.max()))
    assert np.array_equal(a["final_Ts"], b["final_Ts"])
    assert np.array_equal(a["final_idx"], b["final_idx"])
    assert np.abs(a["out_img"] - b["out_img"]).max() <= 2.4e-7  # fma(bg, T, C) vs bg * T + C
    assert abs(loss0 - loss1) <= 1e-7
    for k in GRADS:
        assert rel_l2(b[k], a[k]) <= 1e-6, k


@pytest.mark.parametrize("chunk", [64, 512])
def test_pieces_close_to_one_pass(oracle, chunk):
    g, cam = _long_lists()
    loss0, a = _step(oracle, g, cam, 0)
    loss1, b = _step(oracle, g, cam, chunk)
    assert np.abs(a["out_img"] - b["out_img"]).max() <= 1e-3
    assert abs(loss0 - loss1) <= 1e-5
    for k in GRADS:
        assert rel_l2(b[k], a[k]) <= 5e-2, k
    # the pieces go on past where one pass stops: transmittance only ever lower
    assert np.all(b["final_Ts"] <= a["final_Ts"] + 1e-7)
