"""On-disk formats (CPU): checkpoint v2, PLY and .splat.

PLY and .splat files are compared with the ones the reference's own writers produce
(core/src/loaders/save_gaussians.cpp, compiled into oracle/_ref), and read back with
the reference's reader; the checkpoint layout follows core/src/model.cpp:282-496 and is
checked field by field, through round trips, and on version-1 and sky / exposure
files built here the way the reference writes them.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from msplat_street_b200 import formats, scenes
from oracle_lib import PATHS, available

needs_ref = pytest.mark.skipif(not available("reference_formats"), reason="reference writers not built here")


def _ref():
    lib = C.CDLL(PATHS["reference_formats"])
    lib.ref_save_gaussians.restype = C.c_int
    lib.ref_load_ply.restype = C.c_int
    return lib


def _P(a):
    return C.c_void_p(a.ctypes.data)


def _scene(n=300, deg=3, seed=1):
    g = scenes.random_gaussians(n, seed, sh_degree=deg)
    # quaternions off unit length, as trained ones drift (the .splat writer renormalises)
    g.quats *= np.random.default_rng(seed).uniform(0.5, 2.0, (n, 1)).astype(np.float32)
    return [np.ascontiguousarray(a) for a in g.arrays()]


def _ref_write(tmp_path, params, mode, step=0, scale=1.0, trans=(0.0, 0.0, 0.0), keep=False):
    path = str(tmp_path / ("ref.ply" if mode == 0 else "ref.splat"))
    m, s, q, d, r, o = params
    t = np.asarray(trans, np.float32)
    assert _ref().ref_save_gaussians(path.encode(), mode, m.shape[0], r.shape[1], _P(m), _P(s), _P(q), _P(d),
                                     _P(r), _P(o), step, C.c_float(scale), _P(t), int(keep)) == 0
    return path


@needs_ref
@pytest.mark.parametrize("deg", [3, 0])
def test_ply_bytes_equal_reference(tmp_path, deg):
    params = _scene(deg=deg)
    ref = open(_ref_write(tmp_path, params, 0, step=1234), "rb").read()
    assert formats.ply_bytes(params, step=1234) == ref


@needs_ref
def test_ply_with_crs_matches_reference(tmp_path):
    params = _scene()
    scale, trans = 0.37, (12.5, -3.25, 100.0)
    ref = open(_ref_write(tmp_path, params, 0, 7, scale, trans, True), "rb").read()
    got = formats.ply_bytes(params, 7, scale, trans, True)
    assert len(got) == len(ref)
    hdr = ref.index(b"end_header\n") + len(b"end_header\n")
    assert got[:hdr] == ref[:hdr]
    a = np.frombuffer(got[hdr:], np.float32)
    b = np.frombuffer(ref[hdr:], np.float32)
    # the exponentials may differ in the last place from the reference's float exp
    np.testing.assert_array_max_ulp(a, b, maxulp=2)


@needs_ref
@pytest.mark.parametrize("keep", [False, True])
def test_ply_reader_matches_reference(tmp_path, keep):
    params = _scene(deg=2)
    path = str(tmp_path / "scene.ply")
    formats.save_ply(path, params, step=55)
    scale, trans = (0.5, (1.0, 2.0, 3.0)) if keep else (1.0, (0.0, 0.0, 0.0))
    got, step = formats.load_ply(path, scale, trans, keep)
    lib = _ref()
    t = np.asarray(trans, np.float32)
    n, b, st = C.c_int(), C.c_int(), C.c_int()
    assert lib.ref_load_ply(path.encode(), C.c_float(scale), _P(t), int(keep), C.byref(n), C.byref(b), C.byref(st),
                            None, None, None, None, None, None) == 0
    ref = [np.zeros((n.value, 3), np.float32), np.zeros((n.value, 3), np.float32), np.zeros((n.value, 4), np.float32),
           np.zeros((n.value, 3), np.float32), np.zeros((n.value, b.value, 3), np.float32),
           np.zeros((n.value, 1), np.float32)]
    assert lib.ref_load_ply(path.encode(), C.c_float(scale), _P(t), int(keep), C.byref(n), C.byref(b), C.byref(st),
                            *[_P(a) for a in ref]) == 0
    assert step == st.value == 0  # the reader looks for a comment the writer does not emit
    for i, (x, y) in enumerate(zip(got, ref)):
        if keep and i == 1:
            np.testing.assert_array_max_ulp(x, y, maxulp=2)
        else:
            assert np.array_equal(x, y), i
    if not keep:
        for x, y in zip(got, params):
            assert np.array_equal(x, y.reshape(x.shape))


@needs_ref
@pytest.mark.parametrize("keep", [False, True])
def test_splat_matches_reference(tmp_path, keep):
    params = _scene(n=500)
    scale, trans = (0.25, (3.0, 0.0, -1.0)) if keep else (1.0, (0.0, 0.0, 0.0))
    ref = formats.read_splat(_ref_write(tmp_path, params, 1, 0, scale, trans, keep))
    path = str(tmp_path / "ours.splat")
    formats.save_splat(path, params, scale, trans, keep)
    got = formats.read_splat(path)
    assert got.shape == ref.shape == (500,)
    # same order (sort keys are distinct here), colours and quaternion bytes; positions
    # exact, linear scales within the last place of the exponential
    assert np.array_equal(got["m"], ref["m"])
    np.testing.assert_array_max_ulp(got["s"], ref["s"], maxulp=2)
    assert np.abs(got["c"].astype(int) - ref["c"].astype(int)).max() <= 1
    assert np.array_equal(got["c"][:, :3], ref["c"][:, :3])
    assert np.array_equal(got["q"], ref["q"])


def _ckpt(n=200, seed=0):
    rng = np.random.default_rng(seed)
    p = _scene(n, 3, seed)
    m1 = [rng.normal(size=a.shape).astype(np.float32) for a in p]
    m2 = [rng.random(a.shape).astype(np.float32) for a in p]
    return formats.Checkpoint(1500, 3, 1490, np.array([1.6e-4, 5e-3, 1e-3, 2.5e-3, 1.25e-4, 0.05], np.float32),
                              1.6e-4, 1.6e-6, p, m1, m2)


def test_checkpoint_round_trip(tmp_path):
    ck = _ckpt()
    path = tmp_path / "a.msplat"
    formats.save_checkpoint(path, ck)
    got = formats.load_checkpoint(path)
    assert (got.step, got.sh_degree, got.adam_step, got.num_active) == (1500, 3, 1490, 200)
    assert np.array_equal(got.lrs, ck.lrs) and got.means_lr_init == np.float32(1.6e-4)
    for a, b in zip(got.params + got.exp_avg + got.exp_avg_sq, ck.params + ck.exp_avg + ck.exp_avg_sq):
        assert a.shape == b.shape and np.array_equal(a, b)
    assert got.sky is None and got.exposure is None


def test_checkpoint_layout(tmp_path):
    """Field offsets as Model::saveCheckpoint writes them (core/src/model.cpp:311-371)."""
    ck = _ckpt(n=3)
    path = tmp_path / "b.msplat"
    formats.save_checkpoint(path, ck)
    raw = open(path, "rb").read()
    magic, version, step, num, deg, adam = struct.unpack_from("<IIIIII", raw, 0)
    assert (magic, version, step, num, deg, adam) == (0x4C50534D, 2, 1500, 3, 3, 1490)
    assert np.array_equal(np.frombuffer(raw, np.float32, 6, 24), ck.lrs)
    off = 24 + 24 + 8
    ndim, = struct.unpack_from("<I", raw, off)
    shape = struct.unpack_from("<qq", raw, off + 4)
    nbytes, = struct.unpack_from("<Q", raw, off + 20)
    assert (ndim, shape, nbytes) == (2, (3, 3), 36)
    assert np.array_equal(np.frombuffer(raw, np.float32, 9, off + 28).reshape(3, 3), ck.params[0])
    # 18 arrays, then the two absent-feature flags
    sizes = [a.nbytes + 4 + 8 * a.ndim + 8 for a in ck.params + ck.exp_avg + ck.exp_avg_sq]
    assert len(raw) == off + sum(sizes) + 8
    assert struct.unpack_from("<II", raw, len(raw) - 8) == (0, 0)


def test_checkpoint_version1_and_optional_sections(tmp_path):
    ck = _ckpt(n=10)
    v2 = tmp_path / "v2.msplat"
    formats.save_checkpoint(v2, ck)
    raw = bytearray(open(v2, "rb").read())
    v1 = bytes(raw[:4]) + struct.pack("<I", 1) + bytes(raw[8:-8])  # version 1: no trailing sections
    (tmp_path / "v1.msplat").write_bytes(v1)
    got = formats.load_checkpoint(tmp_path / "v1.msplat")
    assert got.num_active == 10 and np.array_equal(got.params[4], ck.params[4])
    # a v2 file with a learned sky and exposure (written by models that use them) loads;
    # the sections are kept for the caller (the trainer adopts them when it uses them)
    sky = {"frame": np.arange(9, dtype=np.float32), "steps": 77, "tex": np.ones((2, 4, 3), np.float32),
           "exp_avg": np.zeros((2, 4, 3), np.float32), "exp_avg_sq": np.zeros((2, 4, 3), np.float32)}
    expo = {"params": np.ones((5, 4), np.float32), "exp_avg": np.zeros((5, 4), np.float32),
            "exp_avg_sq": np.zeros((5, 4), np.float32), "steps": np.arange(5, dtype=np.int32)}
    ck.sky, ck.exposure = sky, expo
    formats.save_checkpoint(tmp_path / "full.msplat", ck)
    got = formats.load_checkpoint(tmp_path / "full.msplat")
    assert got.sky["steps"] == 77 and np.array_equal(got.sky["frame"], sky["frame"])
    assert np.array_equal(got.exposure["steps"], expo["steps"]) and got.exposure["params"].shape == (5, 4)


def test_checkpoint_rejects_bad_files(tmp_path):
    (tmp_path / "x").write_bytes(b"NOPE" + b"\0" * 60)
    with pytest.raises(ValueError):
        formats.load_checkpoint(tmp_path / "x")
    ck = _ckpt(n=4)
    formats.save_checkpoint(tmp_path / "ok", ck)
    raw = open(tmp_path / "ok", "rb").read()
    (tmp_path / "short").write_bytes(raw[:200])
    with pytest.raises(ValueError):
        formats.load_checkpoint(tmp_path / "short")
    (tmp_path / "v9").write_bytes(raw[:4] + struct.pack("<I", 9) + raw[8:])
    with pytest.raises(ValueError):
        formats.load_checkpoint(tmp_path / "v9")
