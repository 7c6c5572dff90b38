"""Image pipeline, metrics and display kernels against the oracle (needs a GPU).

The reference's tests for this group (tests/test_msplat.py:471-597) check resize,
undistortion, metrics and packing on small synthetic images; here every kernel must
equal the oracle (pinned to the reference backend) bit for bit, on odd sizes,
integer and fractional scale factors, RGBA8 and float sources.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200.backend import Context
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def _img(rng, h, w, c=3):
    return rng.random((h, w, c)).astype(np.float32)


@pytest.mark.parametrize("src_hw,dst_wh", [((37, 53), (20, 14)), ((64, 96), (48, 32)), ((50, 70), (70, 50)),
                                           ((33, 47), (47, 33)), ((720, 1280), (400, 225))])
def test_resize_area_float(oracle, src_hw, dst_wh):
    rng = np.random.default_rng(sum(src_hw))
    a = _img(rng, *src_hw)
    got = Context().resize_area(torch.from_numpy(a).cuda(), *dst_wh).cpu().numpy()
    assert np.array_equal(got, oracle.resize_area(a, *dst_wh))


@pytest.mark.parametrize("src_hw,dst_wh", [((37, 53), (53, 37)), ((37, 53), (17, 11)), ((90, 120), (40, 30))])
def test_resize_area_rgba8(oracle, src_hw, dst_wh):
    rng = np.random.default_rng(7)
    u8 = rng.integers(0, 256, src_hw + (4,)).astype(np.uint8)
    got = Context().resize_area(torch.from_numpy(u8).cuda(), *dst_wh).cpu().numpy()
    assert np.array_equal(got, oracle.resize_area(u8, *dst_wh))


@pytest.mark.parametrize("dist", [[-0.12, 0.03, 0.001, -0.002, 0.004], [0.0, 0.0, 0.0, 0.0, 0.0],
                                  [0.25, -0.1, -0.003, 0.002, 0.01]])
def test_undistort(oracle, dist):
    rng = np.random.default_rng(11)
    a = _img(rng, 61, 83)
    intr = [70.0, 68.5, 41.3, 30.1]
    got = Context().undistort(torch.from_numpy(a).cuda(), intr, dist, 3, 2, 77, 55).cpu().numpy()
    assert np.array_equal(got, oracle.undistort(a, intr, dist, 3, 2, 77, 55))


@pytest.mark.parametrize("hw", [(37, 53), (1, 1), (11, 5), (256, 300)])
def test_image_metrics(oracle, hw):
    rng = np.random.default_rng(hw[0])
    a = _img(rng, *hw)
    b = np.clip(a + rng.normal(0, 0.05, a.shape), 0, 1).astype(np.float32)
    got = np.array(Context().image_metrics(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()))
    assert np.array_equal(got, oracle.image_metrics(a, b))


def test_image_metrics_identical_images_give_infinite_psnr(oracle):
    a = _img(np.random.default_rng(2), 20, 30)
    t = torch.from_numpy(a).cuda()
    psnr, ssim, l1 = Context().image_metrics(t, t)
    assert psnr == float("inf") and l1 == 0.0 and abs(ssim - 1.0) < 1e-6
    assert np.array_equal(np.array([psnr, ssim, l1]), oracle.image_metrics(a, a))


def test_pack_rgba8(oracle):
    rng = np.random.default_rng(4)
    a = (_img(rng, 41, 29) * 1.4 - 0.2).astype(np.float32)  # values beyond [0, 1] clamp
    got = Context().pack_rgba8(torch.from_numpy(a).cuda())
    assert got.shape == (41, 29, 4) and np.array_equal(got, oracle.pack_rgba8(a))


def test_finalize_depth(oracle):
    rng = np.random.default_rng(5)
    t = rng.random(10_000).astype(np.float32)
    t[::13] = 1.0
    t[::17] = 1.0 - 5e-5  # alpha below the 1e-4 cut-off
    dn = (rng.random(10_000) * 4).astype(np.float32)
    d, a = Context().finalize_depth(torch.from_numpy(dn).cuda(), torch.from_numpy(t).cuda(), 0.25)
    od, oa = oracle.finalize_depth(dn, t, 0.25)
    assert np.array_equal(d.cpu().numpy(), od) and np.array_equal(a.cpu().numpy(), oa)


def test_bad_arguments_are_rejected():
    ctx = Context()
    with pytest.raises(ValueError):
        ctx.resize_area(torch.zeros((4, 4, 2), device="cuda"), 2, 2)
    with pytest.raises(ValueError):
        ctx.undistort(torch.zeros((4, 4, 3), device="cuda"), [1, 1, 1], [0] * 5, 0, 0, 2, 2)
