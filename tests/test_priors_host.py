"""Prior-guided training's host side (CPU): prior maps, sky frame and texture set-up,
depth-weight schedule (msplat_street_b200.priors).

Checked against the reference's own code (core/src/priors.cpp, core/src/model.cpp,
compiled into oracle/_ref/libmsplat_ref_priors.so with its loaders) where that build
is present: resampling and prior-map packing bit for bit (files written here and read
by both sides), the sky frame bit for bit, the initial sky texture texel for texel
except where a sample's float asin / atan2 lands on a texel border (the reference
calls the host's float functions, numpy its own).
"""
import ctypes as C
import math

import numpy as np
import pytest

from msplat_street_b200 import priors
from msplat_street_b200.camera import look_at
from oracle_lib import PATHS, available

needs_ref = pytest.mark.skipif(not available("reference_priors"), reason="reference prior code not built here")


def _ref():
    lib = C.CDLL(PATHS["reference_priors"])
    lib.ref_load_priors.restype = C.c_int
    return lib


def _P(a):
    return C.c_void_p(a.ctypes.data)


@needs_ref
@pytest.mark.parametrize("src,dst", [((37, 23), (16, 11)), ((64, 48), (64, 48)), ((13, 7), (40, 30)),
                                     ((1500, 900), (1024, 614))])
def test_resample_nearest_matches_reference(src, dst):
    a = np.random.default_rng(0).random((src[1], src[0])).astype(np.float32)
    ref = np.zeros((dst[1], dst[0]), np.float32)
    _ref().ref_resample_nearest(_P(a), src[0], src[1], _P(ref), dst[0], dst[1])
    assert np.array_equal(priors.resample_nearest(a, dst[0], dst[1]), ref)


def _write_priors(tmp_path, w, h, seed, with_conf=True, with_sky=True, with_mask=True, depth=True):
    from PIL import Image
    rng = np.random.default_rng(seed)
    paths = {"depth": "", "confidence": "", "sky": "", "mask": ""}
    if depth:
        d = (1.0 + 30.0 * rng.random((h, w))).astype(np.float32)
        d[rng.random((h, w)) < 0.05] = 0.0
        d[0, :3] = [np.nan, np.inf, -2.0]
        np.save(tmp_path / "d.npy", d)
        paths["depth"] = str(tmp_path / "d.npy")
        if with_conf:
            c = rng.random((h, w)).astype(np.float64) * 1.2 - 0.1  # out of [0, 1] on purpose
            c[1, 0] = np.nan
            np.save(tmp_path / "c.npy", c)
            paths["confidence"] = str(tmp_path / "c.npy")
    if with_sky:
        s = (rng.random((h, w, 3)) * 255).astype(np.uint8)
        Image.fromarray(s).save(tmp_path / "s.png")
        paths["sky"] = str(tmp_path / "s.png")
    if with_mask:
        m = np.where(rng.random((h, w)) < 0.2, 0, 255).astype(np.uint8)
        Image.fromarray(m).save(tmp_path / "m.png")
        paths["mask"] = str(tmp_path / "m.png")
    return paths


@needs_ref
@pytest.mark.parametrize("case", ["all", "no_conf", "large", "sky_only", "mask_off"])
def test_load_priors_matches_reference(tmp_path, case):
    w, h = (1500, 700) if case == "large" else (97, 61)
    paths = _write_priors(tmp_path, w, h, 3, with_conf=case != "no_conf", depth=case != "sky_only")
    use_mask = case != "mask_off"
    scale = 0.37
    lib = _ref()
    rw, rh = C.c_int(), C.c_int()
    args = [p.encode() for p in (paths["depth"], paths["confidence"], paths["sky"], paths["mask"])]
    assert lib.ref_load_priors(*args, C.c_float(scale), int(use_mask), C.byref(rw), C.byref(rh), None, None,
                               None) == 0
    rd = np.zeros((rh.value, rw.value), np.float32)
    ra = np.zeros((rh.value, rw.value, 4), np.uint8)
    flags = np.zeros(3, np.int32)
    lib.ref_load_priors(*args, C.c_float(scale), int(use_mask), C.byref(rw), C.byref(rh), _P(rd), _P(ra),
                        _P(flags))
    cp = priors.load_camera_prior({k: (v or None) for k, v in paths.items()}, scale, use_mask)
    assert (cp.width, cp.height) == (rw.value, rh.value)
    assert (cp.has_depth, cp.has_sky, cp.has_mask) == tuple(bool(x) for x in flags)
    assert np.array_equal(cp.depth, rd)
    assert np.array_equal(cp.aux, ra)


def test_build_camera_prior_packing():
    d = np.array([[2.0, 0.0], [np.nan, 4.0]], np.float32)
    c = np.array([[0.5, 1.0], [1.0, 2.0]], np.float32)
    sky = np.array([[0.0, 1.0], [0.6, 0.2]], np.float32)
    cp = priors.build_camera_prior(d, c, sky, None, depth_scale=0.5)
    assert np.array_equal(cp.depth, [[1.0, 0.0], [0.0, 2.0]])
    assert cp.aux[..., 0].tolist() == [[128, 0], [0, 255]]  # lround(0.5 * 255) = 128; invalid depth: 0
    assert cp.aux[..., 1].tolist() == [[0, 255], [255, 0]]
    assert (cp.aux[..., 2] == 255).all() and (cp.aux[..., 3] == 0).all()
    assert priors.build_camera_prior(None, None, None, np.ones((2, 2)), use_mask=False) is None


def _poses(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        eye = np.array([2.0 * i, 1.5 + 0.1 * rng.standard_normal(), 0.3 * rng.standard_normal()])
        out.append(look_at(eye, eye + np.array([1.0, 0.05 * rng.standard_normal(), 0.1])).astype(np.float32))
    return out


@needs_ref
@pytest.mark.parametrize("kind", ["street", "looking_up", "degenerate"])
def test_sky_frame_matches_reference(kind):
    if kind == "street":
        poses = _poses(12, 1)
    elif kind == "looking_up":  # headings parallel to the mean up: the fallback axis
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = [[1, 0, 0], [0, 0, 1], [0, -1, 0]]
        poses = [m, m.copy()]
    else:  # ups cancel
        a = np.eye(4, dtype=np.float32)
        b = np.eye(4, dtype=np.float32)
        b[:3, 1] *= -1
        b[:3, 2] *= -1
        poses = [a, b]
    frame = np.zeros(9, np.float32)
    flat = np.ascontiguousarray(np.stack(poses), np.float32)
    _ref().ref_compute_sky_frame(len(poses), _P(flat), _P(frame))
    assert np.array_equal(priors.compute_sky_frame(poses), frame)


class _View:
    def __init__(self, m, w, h, fx, fy, cx, cy, img):
        self.cam_to_world, self.width, self.height = m, w, h
        self.fx, self.fy, self.cx, self.cy, self.image = fx, fy, cx, cy, img


@needs_ref
def test_init_sky_texture_matches_reference():
    rng = np.random.default_rng(4)
    poses = _poses(5, 2)
    views, cps = [], []
    for i, m in enumerate(poses):
        w, h = (640, 360) if i % 2 == 0 else (300, 200)
        img = rng.random((h, w, 3)).astype(np.float32)
        sky = np.zeros((h // 2, w // 2), np.float32)
        sky[: h // 5] = 1.0  # the top rows are sky
        cp = priors.build_camera_prior(None, None, sky, None) if i != 3 else None  # camera 3 has no sky mask
        views.append(_View(m, w, h, 0.8 * w, 0.8 * w, w / 2 + 3.0, h / 2 - 2.0, img))
        cps.append(cp)
    frame = priors.compute_sky_frame(poses)
    W, H = 64, 16
    got = priors.init_sky_texture(views, cps, frame, W, H)
    n = len(views)
    c2w = np.ascontiguousarray(np.stack(poses), np.float32)
    intr = np.array([[v.fx, v.fy, v.cx, v.cy] for v in views], np.float32)
    imgs = (C.c_void_p * n)(*[v.image.ctypes.data for v in views])
    auxs = (C.c_void_p * n)(*[cp.aux.ctypes.data if cp is not None else None for cp in cps])
    has = np.array([int(cp is not None and cp.has_sky) for cp in cps], np.int32)
    sizes = np.array([[v.width, v.height, cp.width if cp else 0, cp.height if cp else 0] for v, cp in
                      zip(views, cps)], np.int32)
    ref = np.zeros((H, W, 3), np.float32)
    _ref().ref_init_sky_texture(n, _P(c2w), _P(intr), imgs, auxs, _P(has), _P(sizes), _P(frame), W, H, _P(ref))
    close = np.isclose(got, ref, rtol=1e-6, atol=1e-7).all(axis=2)
    assert close.mean() >= 0.97, close.mean()
    assert np.abs(got - ref).max() < 0.2  # a border sample moved, nothing else


def test_init_sky_texture_without_sky_is_the_default():
    tex = priors.init_sky_texture([], [], priors.compute_sky_frame([np.eye(4)]), 8, 4)
    assert np.array_equal(tex, np.broadcast_to(np.array([0.6, 0.7, 0.85], np.float32), (4, 8, 3)))


def test_depth_weight_schedule():
    o = priors.PriorOptions(depth_weight=0.1)
    assert priors.depth_weight_at(o, 500, 1000) == pytest.approx(0.1)
    o.depth_weight_final = 0.0
    assert priors.depth_weight_at(o, 250, 1000) == pytest.approx(0.075)
    o.depth_weight_final = 0.001
    assert priors.depth_weight_at(o, 500, 1000) == pytest.approx(math.sqrt(0.1 * 0.001), rel=1e-6)
    assert priors.depth_weight_at(o, 5000, 1000) == pytest.approx(0.001, rel=1e-6)
    assert priors.depth_weight_at(priors.PriorOptions(), 10, 100) == 0.0
    assert not priors.PriorOptions().active() and priors.PriorOptions(max_scale_ratio=2.0).active()


def test_prior_paths(tmp_path):
    for sub, name in (("depth", "cam0/0001.npy"), ("sky", "0001.png"), ("mask", "cam0/0001.jpg")):
        p = tmp_path / sub / name
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(b"x")
    got = priors.prior_paths("cam0/0001.jpg", str(tmp_path))
    assert got["depth"].endswith("depth/cam0/0001.npy") and got["sky"].endswith("sky/0001.png")
    assert got["mask"].endswith("mask/cam0/0001.jpg") and got["confidence"] is None
