"""On-disk formats of trained scenes: the msplat checkpoint, PLY and .splat.

* Checkpoint v2 (``.msplat``; core/src/model.cpp:282-496): magic "MSPL", version, the
  step / active count / SH degree / Adam step, the six learning rates and the means
  schedule, the six parameter arrays, both Adam moments per group, then the learned
  sky and per-image exposure sections (present flags; written when the trainer uses
  them, adopted on load only by a trainer configured with the same shapes, as
  Model::loadCheckpoint does).
  Every array is ndim (u32), shape (i64 each), byte count (u64), float32 data.
* PLY (core/src/loaders/save_gaussians.cpp:10-53 writer, :112-190 reader): the 3DGS
  layout -- xyz, zero normals, f_dc, f_rest transposed to (3, bases), opacity logit,
  log-scales, quaternion -- optionally mapped back to a source CRS (scale,
  translation).
* .splat (:56-110): 32-byte records (position, linear scale, RGBA8 colour,
  quaternion as bytes), largest / most opaque first.

Files written here are byte-identical to the reference's where no exponential is
involved; the exponentials (CRS-mapped scales, .splat scales, sort keys and alpha) are
evaluated in float64 and rounded once, which equals the reference's float ``exp`` on
all but rare last-place ties.
"""
from __future__ import annotations

import io
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

CKPT_MAGIC = 0x4C50534D  # "MSPL"
CKPT_VERSION = 2
N_ADAM_GROUPS = 6
SH_C0 = 0.28209479177387814


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float32))


def _exp32(x: np.ndarray) -> np.ndarray:
    return np.exp(np.asarray(x, np.float64)).astype(np.float32)


def _log32(x: np.ndarray) -> np.ndarray:
    return np.log(np.asarray(x, np.float64)).astype(np.float32)


# ---- checkpoint ----------------------------------------------------------------------

@dataclass
class Checkpoint:
    """The state Model::saveCheckpoint stores (core/src/model.cpp:311-371)."""

    step: int
    sh_degree: int
    adam_step: int
    lrs: np.ndarray  # (6,) float32: means, scales, quats, dc, rest, opacity
    means_lr_init: float
    means_lr_final: float
    params: List[np.ndarray]  # means (N,3), scales (N,3), quats (N,4), dc (N,3), rest (N,B-1,3), opacities (N,1)
    exp_avg: List[np.ndarray]
    exp_avg_sq: List[np.ndarray]
    sky: Optional[dict] = None  # frame (9,), steps, tex, exp_avg, exp_avg_sq
    exposure: Optional[dict] = None  # params, exp_avg, exp_avg_sq, steps

    @property
    def num_active(self) -> int:
        return int(self.params[0].shape[0])


def _write_tensor(f, a: np.ndarray) -> None:
    a = _f32(a)
    f.write(struct.pack("<I", a.ndim))
    for s in a.shape:
        f.write(struct.pack("<q", int(s)))
    f.write(struct.pack("<Q", a.nbytes))
    f.write(a.tobytes())


def _read_exact(f, n: int) -> bytes:
    b = f.read(n)
    if len(b) != n:
        raise ValueError("truncated checkpoint")
    return b


def _read_tensor(f) -> np.ndarray:
    (ndim,) = struct.unpack("<I", _read_exact(f, 4))
    if ndim > 8:
        raise ValueError(f"corrupt tensor header (ndim {ndim})")
    shape = [struct.unpack("<q", _read_exact(f, 8))[0] for _ in range(ndim)]
    (nbytes,) = struct.unpack("<Q", _read_exact(f, 8))
    if any(s < 0 for s in shape) or nbytes != 4 * int(np.prod(shape, dtype=np.int64)):
        raise ValueError(f"corrupt tensor header (shape {shape}, {nbytes} bytes)")
    return np.frombuffer(_read_exact(f, nbytes), np.float32).reshape(shape).copy()


def save_checkpoint(path, ck: Checkpoint) -> None:
    """Model::saveCheckpoint's layout (core/src/model.cpp:311-371)."""
    with open(path, "wb") as f:
        f.write(struct.pack("<II", CKPT_MAGIC, CKPT_VERSION))
        f.write(struct.pack("<IIII", ck.step, ck.num_active, ck.sh_degree, ck.adam_step))
        f.write(_f32(ck.lrs).reshape(N_ADAM_GROUPS).tobytes())
        f.write(struct.pack("<ff", ck.means_lr_init, ck.means_lr_final))
        for a in ck.params:
            _write_tensor(f, a)
        for a in ck.exp_avg:
            _write_tensor(f, a)
        for a in ck.exp_avg_sq:
            _write_tensor(f, a)
        if ck.sky is not None:
            f.write(struct.pack("<I", 1))
            f.write(_f32(ck.sky["frame"]).reshape(9).tobytes())
            f.write(struct.pack("<i", int(ck.sky["steps"])))
            for k in ("tex", "exp_avg", "exp_avg_sq"):
                _write_tensor(f, ck.sky[k])
        else:
            f.write(struct.pack("<I", 0))
        if ck.exposure is not None:
            f.write(struct.pack("<I", 1))
            for k in ("params", "exp_avg", "exp_avg_sq"):
                _write_tensor(f, ck.exposure[k])
            steps = np.asarray(ck.exposure["steps"], np.int32)
            f.write(struct.pack("<I", steps.size))
            f.write(steps.tobytes())
        else:
            f.write(struct.pack("<I", 0))


def load_checkpoint(path) -> Checkpoint:
    """Model::loadCheckpoint (core/src/model.cpp:373-496): versions 1 and 2."""
    with open(path, "rb") as f:
        magic, version = struct.unpack("<II", _read_exact(f, 8))
        if magic != CKPT_MAGIC:
            raise ValueError("Not a valid msplat checkpoint file")
        if version < 1 or version > CKPT_VERSION:
            raise ValueError(f"Unsupported checkpoint version: {version}")
        step, num, deg, adam_step = struct.unpack("<IIII", _read_exact(f, 16))
        lrs = np.frombuffer(_read_exact(f, 4 * N_ADAM_GROUPS), np.float32).copy()
        lr0, lr1 = struct.unpack("<ff", _read_exact(f, 8))
        params = [_read_tensor(f) for _ in range(6)]
        m1 = [_read_tensor(f) for _ in range(N_ADAM_GROUPS)]
        m2 = [_read_tensor(f) for _ in range(N_ADAM_GROUPS)]
        sky = expo = None
        if version >= 2:
            (has_sky,) = struct.unpack("<I", _read_exact(f, 4))
            if has_sky:
                frame = np.frombuffer(_read_exact(f, 36), np.float32).copy()
                (steps,) = struct.unpack("<i", _read_exact(f, 4))
                tex, ea, eas = _read_tensor(f), _read_tensor(f), _read_tensor(f)
                sky = {"frame": frame, "steps": steps, "tex": tex, "exp_avg": ea, "exp_avg_sq": eas}
            (has_expo,) = struct.unpack("<I", _read_exact(f, 4))
            if has_expo:
                p, ea, eas = _read_tensor(f), _read_tensor(f), _read_tensor(f)
                (n,) = struct.unpack("<I", _read_exact(f, 4))
                steps = np.frombuffer(_read_exact(f, 4 * n), np.int32).copy()
                expo = {"params": p, "exp_avg": ea, "exp_avg_sq": eas, "steps": steps}
    if params[0].shape[0] != num:
        raise ValueError(f"checkpoint says {num} Gaussians, arrays hold {params[0].shape[0]}")
    return Checkpoint(step, deg, adam_step, lrs, lr0, lr1, params, m1, m2, sky, expo)


# ---- PLY --------------------------------------------------------------------------

def _crs_out(means, scales, scale, translation, keep_crs):
    if not keep_crs:
        return _f32(means), _f32(scales)
    s = np.float32(scale)
    t = _f32(translation).reshape(1, 3)
    return (_f32(means) / s + t).astype(np.float32), _log32(_exp32(scales) / s)


def ply_bytes(params: Sequence[np.ndarray], step: int = 0, scale: float = 1.0, translation=(0.0, 0.0, 0.0),
              keep_crs: bool = False) -> bytes:
    """saveGaussianPly (core/src/loaders/save_gaussians.cpp:10-53) as bytes."""
    means, scales, quats, dc, rest, opac = [_f32(a) for a in params]
    n = means.shape[0]
    rest = rest.reshape(n, -1, 3)
    num_dc, bases = dc.reshape(n, -1).shape[1], rest.shape[1]
    hdr = io.StringIO()
    hdr.write("ply\nformat binary_little_endian 1.0\n")
    hdr.write(f"comment msplat v{step}\n")
    hdr.write(f"element vertex {n}\n")
    hdr.write("property float x\nproperty float y\nproperty float z\n")
    hdr.write("property float nx\nproperty float ny\nproperty float nz\n")
    for i in range(num_dc):
        hdr.write(f"property float f_dc_{i}\n")
    for i in range(bases * 3):
        hdr.write(f"property float f_rest_{i}\n")
    hdr.write("property float opacity\n")
    hdr.write("property float scale_0\nproperty float scale_1\nproperty float scale_2\n")
    hdr.write("property float rot_0\nproperty float rot_1\nproperty float rot_2\nproperty float rot_3\n")
    hdr.write("end_header\n")
    m, s = _crs_out(means, scales, scale, translation, keep_crs)
    rows = np.concatenate([m, np.zeros((n, 3), np.float32), dc.reshape(n, num_dc),
                           rest.transpose(0, 2, 1).reshape(n, 3 * bases),  # PLY keeps (3, bases) per row
                           opac.reshape(n, 1), s, quats.reshape(n, 4)], axis=1).astype(np.float32)
    return hdr.getvalue().encode("ascii") + np.ascontiguousarray(rows).tobytes()


def save_ply(path, params: Sequence[np.ndarray], step: int = 0, scale: float = 1.0, translation=(0.0, 0.0, 0.0),
             keep_crs: bool = False) -> None:
    with open(path, "wb") as f:
        f.write(ply_bytes(params, step, scale, translation, keep_crs))


def load_ply(path, scale: float = 1.0, translation=(0.0, 0.0, 0.0), keep_crs: bool = False):
    """loadGaussianPly (core/src/loaders/save_gaussians.cpp:112-190): returns
    (params, step) with params in the backend's layouts."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.find(b"end_header\n")
    if not data.startswith(b"ply") or end < 0:
        raise ValueError(f"Not a PLY file: {path}")
    n = step = num_dc = num_fr = 0
    for line in data[:end].decode("ascii", "replace").split("\n"):
        if line.startswith("comment Generated by msplat at iteration "):
            step = int(line[len("comment Generated by msplat at iteration "):])
        elif line.startswith("element vertex "):
            n = int(line[len("element vertex "):])
        elif line.startswith("property float f_dc_"):
            num_dc += 1
        elif line.startswith("property float f_rest_"):
            num_fr += 1
    if n == 0:
        raise ValueError("PLY has no vertices")
    cols = 3 + 3 + num_dc + num_fr + 1 + 3 + 4
    body = data[end + len(b"end_header\n"):]
    if len(body) < n * cols * 4:
        raise ValueError("PLY body is shorter than its header says")
    rows = np.frombuffer(body[:n * cols * 4], np.float32).reshape(n, cols)
    c = 0
    means = rows[:, c:c + 3].copy(); c += 6  # xyz, then the unused normals
    dc = rows[:, c:c + num_dc].copy(); c += num_dc
    bases = num_fr // 3
    rest = rows[:, c:c + num_fr].reshape(n, 3, bases).transpose(0, 2, 1).copy(); c += num_fr
    opac = rows[:, c:c + 1].copy(); c += 1
    scales = rows[:, c:c + 3].copy(); c += 3
    quats = rows[:, c:c + 4].copy()
    if keep_crs:
        t = _f32(translation).reshape(1, 3)
        means = ((means - t) * np.float32(scale)).astype(np.float32)
        scales = _log32(np.float32(scale) * _exp32(scales))
    return [means, scales, quats, dc, np.ascontiguousarray(rest), opac], step


# ---- .splat ----------------------------------------------------------------------

def splat_bytes(params: Sequence[np.ndarray], scale: float = 1.0, translation=(0.0, 0.0, 0.0),
                keep_crs: bool = False) -> bytes:
    """saveGaussianSplat (core/src/loaders/save_gaussians.cpp:56-110) as bytes."""
    means, scales, quats, dc, _, opac = [_f32(a) for a in params]
    n = means.shape[0]
    es = _exp32(scales)
    size = (es[:, 0] + es[:, 1]) + es[:, 2]
    if keep_crs:
        size = (size / np.float32(scale)).astype(np.float32)
    sig_den = (np.float32(1.0) + _exp32(-opac.reshape(n))).astype(np.float32)
    key = (size / sig_den).astype(np.float32)
    order = np.argsort(-key, kind="stable")  # largest first
    m, _ = _crs_out(means, scales, scale, translation, keep_crs)
    sc = (es / np.float32(scale)).astype(np.float32) if keep_crs else es
    rgb = np.clip((dc.astype(np.float64) * SH_C0 + 0.5) * 255.0, 0.0, 255.0).astype(np.uint8)
    sig = (np.float32(1.0) / sig_den).astype(np.float32)
    alpha = np.clip(sig * np.float32(255.0), 0.0, 255.0).astype(np.uint8)
    q = quats.reshape(n, 4)
    qn = np.sqrt(((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3]).astype(np.float32)
    unit = np.where(qn[:, None] > 0, q / np.where(qn > 0, qn, 1)[:, None],
                    np.array([1.0, 0.0, 0.0, 0.0], np.float32)).astype(np.float32)
    qb = np.clip(unit * np.float32(128.0) + np.float32(128.0), 0.0, 255.0).astype(np.uint8)
    rec = np.zeros(n, dtype=[("m", "<f4", 3), ("s", "<f4", 3), ("c", "u1", 4), ("q", "u1", 4)])
    rec["m"] = m
    rec["s"] = sc
    rec["c"][:, :3] = rgb
    rec["c"][:, 3] = alpha.reshape(n)
    rec["q"] = qb
    return rec[order].tobytes()


def save_splat(path, params: Sequence[np.ndarray], scale: float = 1.0, translation=(0.0, 0.0, 0.0),
               keep_crs: bool = False) -> None:
    with open(path, "wb") as f:
        f.write(splat_bytes(params, scale, translation, keep_crs))


def read_splat(path) -> np.ndarray:
    """The 32-byte records of a .splat file (fields m, s, c, q)."""
    return np.fromfile(path, dtype=[("m", "<f4", 3), ("s", "<f4", 3), ("c", "u1", 4), ("q", "u1", 4)])
