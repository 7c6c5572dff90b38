"""ctypes access to the parity oracles (test infrastructure).

``Oracle("restatement")`` loads oracle/_build/libmsplat_oracle.so (this repository's
CPU restatement of the reference backend); ``Oracle("reference")`` loads
oracle/_ref/libmsplat_ref.so (the reference's own core/cpu backend, built by
oracle/Makefile where the reference sources are present). Both export the C-ABI in
oracle/msplat_oracle.h, so every test can run against either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
PATHS = {
    "restatement": os.path.join(ORACLE_DIR, "_build", "libmsplat_oracle.so"),
    "reference": os.path.join(ORACLE_DIR, "_ref", "libmsplat_ref.so"),
    "reference_fast": os.path.join(ORACLE_DIR, "_ref", "libmsplat_ref_fast.so"),
    "reference_formats": os.path.join(ORACLE_DIR, "_ref", "libmsplat_ref_formats.so"),
    "reference_priors": os.path.join(ORACLE_DIR, "_ref", "libmsplat_ref_priors.so"),
    "reference_model": os.path.join(ORACLE_DIR, "_ref", "libmsplat_ref_model.so"),
}

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_FRAME_DTYPES = {"radii": np.int32, "tile_start": np.int32, "tile_end": np.int32, "isect_gid": np.int32,
                 "final_idx": np.int32, "chunk_first": np.int32}


def available(kind: str) -> bool:
    return os.path.exists(PATHS[kind])


def build_restatement() -> None:
    """Compile the restatement if it is missing (needs only g++)."""
    if not available("restatement"):
        subprocess.run(["make", "-C", ORACLE_DIR, "_build/libmsplat_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)


def P(a):
    """Pointer to a numpy array's data, typed so ctypes passes all 64 bits."""
    return C.c_void_p(a.ctypes.data)


def _ptr_array(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class Oracle:
    def __init__(self, kind: str = "restatement"):
        if kind == "restatement":
            build_restatement()
        path = PATHS[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind = kind
        self.lib = lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        lib.orc_render.restype = C.c_int
        lib.orc_train_step.restype = C.c_float
        lib.orc_frame.restype = C.c_int64
        lib.orc_frame.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        lib.orc_densify.restype = C.c_int

    # -- rendering and training ------------------------------------------------

    @staticmethod
    def _cam_args(cam, degree, dtu, clip=0.01):
        return [P(cam.viewmat), P(cam.projmat), C.c_float(cam.fx), C.c_float(cam.fy),
                C.c_float(cam.cx), C.c_float(cam.cy), C.c_uint(cam.height), C.c_uint(cam.width),
                C.c_int(cam.tiles_x), C.c_int(cam.tiles_y), C.c_float(clip), C.c_uint(degree), C.c_uint(dtu),
                P(cam.cam_pos)]

    def render(self, g, cam, bg, degrees_to_use=None, glob_scale=1.0):
        deg = g.sh_degree
        dtu = deg if degrees_to_use is None else degrees_to_use
        out = np.zeros((cam.height, cam.width, 3), np.float32)
        bg = np.ascontiguousarray(bg, np.float32)
        args = [C.c_int(g.n), P(g.means), P(g.scales), C.c_float(glob_scale), P(g.quats)]
        args += self._cam_args(cam, deg, dtu)
        args += [P(g.features_dc), P(g.features_rest), P(g.opacities), P(bg),
                 P(out)]
        self.lib.orc_render(*args)
        return out

    def train_step(self, g, cam, bg, gt, adam, stats, ssim_weight=0.2, degrees_to_use=None, glob_scale=1.0):
        """One msplat_train_step; ``g``, ``adam`` (dict with m1, m2 lists, step_sizes,
        bc2, beta1, beta2, eps) and ``stats`` (vis, gn, ms) are updated in place."""
        deg = g.sh_degree
        dtu = deg if degrees_to_use is None else degrees_to_use
        bg = np.ascontiguousarray(bg, np.float32)
        gt = np.ascontiguousarray(gt, np.float32)
        numel = np.array([a.size for a in g.arrays()], np.int64)
        ss = np.asarray(adam["step_sizes"], np.float32)
        bc2 = np.asarray(adam["bc2"], np.float32)
        args = [C.c_int(g.n), P(g.means), P(g.scales), C.c_float(glob_scale), P(g.quats)]
        args += self._cam_args(cam, deg, dtu)
        args += [P(g.features_dc), P(g.features_rest), P(g.opacities), P(bg),
                 P(gt), C.c_float(ssim_weight), C.c_float(1.0 / (cam.width * cam.height * 3)),
                 _ptr_array(adam["m1"]), _ptr_array(adam["m2"]), P(numel), P(ss),
                 P(bc2), C.c_float(adam["beta1"]), C.c_float(adam["beta2"]), C.c_float(adam["eps"]),
                 P(stats["vis"]), P(stats["gn"]), P(stats["ms"]),
                 C.c_float(1.0 / max(cam.width, cam.height))]
        return float(self.lib.orc_train_step(*args))

    def frame(self, name):
        p = C.c_void_p()
        n = self.lib.orc_frame(name.encode(), C.byref(p))
        if n < 0:
            raise KeyError(name)
        dt = _FRAME_DTYPES.get(name, np.float32)
        if n == 0 or not p.value:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), shape=(n,)).copy()

    # -- densification, primitives, init ----------------------------------------

    def densify(self, n, cap, bufs, m1, m2, stats, half_max_dim, seed, grad_thresh=2e-4, size_thresh=0.01,
                screen_thresh=0.05, check_screen=1, cull_alpha=0.1, cull_scale=0.5, cull_screen=0.15,
                check_huge=1):
        fr_stride = bufs[4].size // cap
        r = self.lib.orc_densify(
            C.c_int(n), C.c_int(cap), C.c_float(grad_thresh), C.c_float(size_thresh), C.c_float(screen_thresh),
            C.c_int(check_screen), C.c_float(cull_alpha), C.c_float(cull_scale), C.c_float(cull_screen),
            C.c_int(check_huge), P(stats["gn"]), P(stats["vis"]), P(stats["ms"]),
            C.c_float(half_max_dim), *[P(b) for b in bufs], C.c_int(fr_stride), _ptr_array(m1),
            _ptr_array(m2), C.c_uint32(seed))
        return int(r)

    def opacity_reset(self, opac, m1, m2, n, reset_logit):
        self.lib.orc_opacity_reset(P(opac), P(m1), P(m2), C.c_int(n),
                                   C.c_float(reset_logit))

    def radix_sort(self, keys, key_bits):
        keys = np.ascontiguousarray(keys, np.uint64).copy()
        vals = np.arange(keys.size, dtype=np.int32)
        self.lib.orc_radix_sort(P(keys), P(vals), C.c_uint32(keys.size), C.c_int(key_bits))
        return keys, vals

    def knn3_mean_dist(self, pts):
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.zeros(pts.shape[0], np.float32)
        self.lib.orc_knn3_mean_dist(P(pts), C.c_uint32(pts.shape[0]), P(out))
        return out

    def init_gaussians(self, pts, rgb, seed, opacity_logit):
        n = pts.shape[0]
        pts = np.ascontiguousarray(pts, np.float32)
        rgb = np.ascontiguousarray(rgb, np.uint8)
        s = np.zeros((n, 3), np.float32)
        q = np.zeros((n, 4), np.float32)
        d = np.zeros((n, 3), np.float32)
        o = np.zeros((n, 1), np.float32)
        self.lib.orc_init_gaussians(P(pts), P(rgb), C.c_uint32(n), C.c_uint32(seed),
                                    C.c_float(opacity_logit), P(s), P(q), P(d),
                                    P(o))
        return s, q, d, o

    # -- image pipeline --------------------------------------------------------

    def resize_area(self, img, out_w, out_h):
        img = np.ascontiguousarray(img)
        u8 = img.dtype == np.uint8
        out = np.zeros((out_h, out_w, 3), np.float32)
        self.lib.orc_resize_area(P(img), C.c_int(int(u8)), C.c_int(img.shape[1]), C.c_int(img.shape[0]),
                                 P(out), C.c_int(out_w), C.c_int(out_h))
        return out

    def image_metrics(self, a, b):
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        out = np.zeros(3, np.float64)
        self.lib.orc_image_metrics(P(a), P(b), C.c_int(a.shape[0]), C.c_int(a.shape[1]),
                                   P(out))
        return out

    def pack_rgba8(self, img):
        img = np.ascontiguousarray(img, np.float32)
        n = img.size // 3
        out = np.zeros(img.shape[:-1] + (4,), np.uint8)
        self.lib.orc_pack_rgba8(P(img), C.c_uint32(n), P(out))
        return out

    def undistort(self, img, intr, dist, roi_x, roi_y, out_w, out_h):
        img = np.ascontiguousarray(img, np.float32)
        it = np.ascontiguousarray(intr, np.float32)
        ds = np.ascontiguousarray(dist, np.float32)
        out = np.zeros((out_h, out_w, 3), np.float32)
        self.lib.orc_undistort(P(img), C.c_int(img.shape[1]), C.c_int(img.shape[0]), P(it), P(ds), C.c_int(roi_x),
                               C.c_int(roi_y), P(out), C.c_int(out_w), C.c_int(out_h))
        return out

    def finalize_depth(self, depth_num, final_t, inv_scale):
        d = np.ascontiguousarray(depth_num, np.float32)
        t = np.ascontiguousarray(final_t, np.float32)
        od, oa = np.zeros_like(d), np.zeros_like(t)
        self.lib.orc_finalize_depth(P(d), P(t), C.c_uint32(d.size), C.c_float(inv_scale), P(od), P(oa))
        return od, oa


def new_adam_state(g, lrs, step: int, beta1=0.9, beta2=0.999, eps=1e-8):
    """Moments and the step sizes Model::fullIteration derives (core/src/model.cpp:638-651)."""
    bc1 = np.float32(1.0 - float(np.float32(beta1)) ** int(step))
    bc2 = np.float32(1.0 - float(np.float32(beta2)) ** int(step))
    return {
        "m1": [np.zeros_like(a) for a in g.arrays()],
        "m2": [np.zeros_like(a) for a in g.arrays()],
        "step_sizes": [np.float32(lr) / bc1 for lr in lrs],
        "bc2": [np.float32(np.sqrt(bc2))] * 6,
        "beta1": beta1, "beta2": beta2, "eps": eps,
    }


def set_option(oracle: "Oracle", name: str, value: int) -> None:
    """Restatement-only switches (see orc_set_option in oracle/msplat_oracle.h)."""
    fn = getattr(oracle.lib, "orc_set_option", None)
    if fn is None or fn(name.encode(), C.c_int(value)) != 0:
        raise KeyError(f"{oracle.kind} oracle has no option {name}")


class OrcPrior(C.Structure):
    """oracle/msplat_oracle.h orc_prior (core/metal/bindings.h:43-77, PriorStep)."""
    _fields_ = [("aux", C.c_int), ("sky", C.c_int),
                ("sky_tex", C.c_void_p), ("sky_grad", C.c_void_p), ("sky_exp_avg", C.c_void_p),
                ("sky_exp_avg_sq", C.c_void_p), ("sky_w", C.c_int), ("sky_h", C.c_int),
                ("sky_frame", C.c_float * 9), ("sky_step_size", C.c_float), ("sky_bc2_sqrt", C.c_float),
                ("prior_depth", C.c_void_p), ("prior_aux", C.c_void_p), ("prior_w", C.c_int), ("prior_h", C.c_int),
                ("has_depth", C.c_int), ("has_sky_mask", C.c_int), ("depth_weight", C.c_float),
                ("sky_weight", C.c_float), ("fill_weight", C.c_float), ("huber_delta", C.c_float),
                ("min_alpha", C.c_float), ("mask_photometric", C.c_int), ("loss_terms", C.c_void_p),
                ("exposure", C.c_int), ("cam_index", C.c_int), ("expo_params", C.c_void_p),
                ("expo_exp_avg", C.c_void_p), ("expo_exp_avg_sq", C.c_void_p), ("expo_grad", C.c_void_p),
                ("expo_step_size", C.c_float), ("expo_bc2_sqrt", C.c_float), ("expo_reg", C.c_float),
                ("log_max_scale_ratio", C.c_float)]


_PRIOR_ARRAYS = ("sky_tex", "sky_grad", "sky_exp_avg", "sky_exp_avg_sq", "prior_depth", "prior_aux", "loss_terms",
                 "expo_params", "expo_exp_avg", "expo_exp_avg_sq", "expo_grad")


def orc_prior(pr: dict) -> OrcPrior:
    """An OrcPrior over the numpy arrays of a prior dict (the arrays must outlive it)."""
    s = OrcPrior()
    for name, _ in OrcPrior._fields_:
        if name in _PRIOR_ARRAYS:
            a = pr.get(name)
            setattr(s, name, None if a is None else a.ctypes.data)
        elif name == "sky_frame":
            s.sky_frame[:] = [float(v) for v in np.asarray(pr.get("sky_frame", np.zeros(9)), np.float32)]
        elif name in pr:
            setattr(s, name, pr[name])
    return s


def set_prior(oracle: "Oracle", pr) -> None:
    """orc_set_prior: ``pr`` (a dict as tests/prior_util.py builds, or None) applies to
    every later render / train step of this oracle."""
    oracle._prior = None if pr is None else orc_prior(pr)
    oracle.lib.orc_set_prior(None if pr is None else C.byref(oracle._prior))
