"""ctypes binding of libmsplat_cuda.so (include/msplat_cuda.h).

This is the product path: there is no CPU fallback. Loading fails loudly when the
library has not been built or no CUDA device is present, and every non-zero status
from the library raises ``MsplatCudaError`` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmsplat_cuda.so")

_STATUS = {1: ValueError, 2: RuntimeError, 3: RuntimeError, 4: OverflowError, 5: NotImplementedError}


class MsplatCudaError(RuntimeError):
    pass


_lib = None

vp = C.c_void_p
f32 = C.c_float
i32 = C.c_int
u32 = C.c_uint
i64 = C.c_int64
sz = C.c_size_t
PP = C.POINTER(C.c_void_p)

_SIGS = {
    "msplat_cuda_last_error": (C.c_char_p, []),
    "msplat_cuda_version": (i32, []),
    "msplat_cuda_ctx_create": (i32, [PP]),
    "msplat_cuda_ctx_destroy": (None, [vp]),
    "msplat_cuda_default_ctx": (vp, []),
    "msplat_cuda_ctx_set_stream": (i32, [vp, vp]),
    "msplat_cuda_ctx_set_option": (i32, [vp, C.c_char_p, i64]),
    "msplat_cuda_cleanup": (i32, [vp]),
    "msplat_cuda_commit": (i32, [vp]),
    "msplat_cuda_sync": (i32, [vp]),
    "msplat_cuda_alloc": (i32, [sz, i32, PP]),
    "msplat_cuda_free": (i32, [vp]),
    "msplat_cuda_copy_buffer": (i32, [vp, vp, vp, sz]),
    "msplat_cuda_render": (i32, [vp, i32, vp, vp, f32, vp, vp, vp, f32, f32, f32, f32, u32, u32, i32, i32, f32, u32,
                                 u32, vp, vp, vp, vp, vp, PP]),
    "msplat_cuda_train_step": (i32, [vp, i32, vp, vp, f32, vp, vp, vp, f32, f32, f32, f32, u32, u32, i32, i32, f32,
                                     u32, u32, vp, vp, vp, vp, vp, vp, f32, f32, i32, vp, vp, vp, vp, f32, f32, f32,
                                     vp, vp, vp, f32, PP, vp]),
    "msplat_cuda_densify": (i32, [vp, i32, i32, f32, f32, f32, i32, f32, f32, f32, i32, vp, vp, vp, f32, vp, i32, vp,
                                  vp, C.c_uint32, C.POINTER(i32)]),
    "msplat_cuda_opacity_reset": (i32, [vp, vp, vp, vp, i32, f32]),
    "msplat_cuda_radix_sort": (i32, [vp, vp, vp, C.c_uint32, i32]),
    "msplat_cuda_radix_sort_static": (i32, [vp, vp, vp, C.c_uint32, i32]),
    "msplat_cuda_knn3_mean_dist": (i32, [vp, vp, C.c_uint32, vp]),
    "msplat_cuda_init_gaussians": (i32, [vp, vp, vp, C.c_uint32, C.c_uint32, f32, vp, vp, vp, vp]),
    "msplat_cuda_render_backward": (i32, [vp, i32, vp, vp, f32, vp, vp, vp, f32, f32, f32, f32, u32, u32, i32, i32,
                                          f32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "msplat_cuda_ssim_loss": (i32, [vp, vp, vp, u32, u32, f32, f32, vp, vp]),
    "msplat_cuda_loss_device": (i32, [vp, PP]),
    "msplat_cuda_frame": (i32, [vp, C.c_char_p, PP, C.POINTER(i64)]),
    "msplat_cuda_num_isects": (i64, [vp]),
    "msplat_cuda_frame_pair_counts": (i32, [vp, vp]),
    "msplat_cuda_frame_pair_counts_device": (i32, [vp, vp]),
    "msplat_cuda_device_alloc": (i32, [sz, PP]),
    "msplat_cuda_rasterizer_exp": (i32, [vp, vp, i64, vp]),
    "msplat_cuda_ctx_device_bytes": (i64, [vp]),
    "msplat_cuda_drain_stage_times": (i32, [vp, vp, vp, i32, C.POINTER(i32), vp]),
}

class View(C.Structure):
    """msplat_cuda_view (include/msplat_cuda.h): one view of a batched render."""
    _fields_ = [
        ("num_points", C.c_int32),
        ("means3d", vp), ("scales", vp), ("quats", vp), ("features_dc", vp), ("features_rest", vp),
        ("opacities", vp),
        ("glob_scale", f32),
        ("degree", C.c_uint32), ("degrees_to_use", C.c_uint32),
        ("viewmat", f32 * 16), ("projmat", f32 * 16),
        ("fx", f32), ("fy", f32), ("cx", f32), ("cy", f32),
        ("img_height", C.c_uint32), ("img_width", C.c_uint32),
        ("clip_thresh", f32),
        ("cam_pos", f32 * 3),
        ("background", f32 * 3),
        ("out_img", vp),
    ]


_SIGS["msplat_cuda_render_batch"] = (i32, [vp, C.c_int32, C.POINTER(View)])


class TrainView(C.Structure):
    """msplat_cuda_train_view (include/msplat_cuda.h): one view of a batched step."""
    _fields_ = [
        ("viewmat", f32 * 16), ("projmat", f32 * 16),
        ("fx", f32), ("fy", f32), ("cx", f32), ("cy", f32),
        ("img_height", C.c_uint32), ("img_width", C.c_uint32),
        ("cam_pos", f32 * 3),
        ("gt", vp),
    ]


_SIGS["msplat_cuda_train_batch"] = (i32, [vp, i32, vp, vp, f32, vp, vp, vp, vp, u32, u32, f32, vp, C.c_int32,
                                          C.POINTER(TrainView), f32, i32, vp, vp, vp, vp, f32, f32, f32, vp, vp, vp,
                                          vp, vp])
_SIGS["msplat_cuda_train_batch_stats"] = (i32, [vp, C.POINTER(i64)])
_SIGS["msplat_cuda_raster_variant"] = (i32, [i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32)])
_SIGS["msplat_cuda_raster_shape"] = (i32, [i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)])
_SIGS["msplat_cuda_resize_area"] = (i32, [vp, vp, i32, i32, i32, vp, i32, i32])
_SIGS["msplat_cuda_undistort"] = (i32, [vp, vp, i32, i32, vp, vp, i32, i32, vp, i32, i32])
_SIGS["msplat_cuda_image_metrics"] = (i32, [vp, vp, vp, i32, i32, vp])
_SIGS["msplat_cuda_pack_rgba8"] = (i32, [vp, vp, C.c_uint32, vp])
_SIGS["msplat_cuda_finalize_depth"] = (i32, [vp, vp, vp, C.c_uint32, f32, vp, vp])


class Prior(C.Structure):
    """msplat_cuda_prior (include/msplat_cuda.h; PriorStep, core/metal/bindings.h:43-77)."""
    _fields_ = [
        ("aux", C.c_int32), ("sky", C.c_int32),
        ("sky_tex", vp), ("sky_grad", vp), ("sky_exp_avg", vp), ("sky_exp_avg_sq", vp),
        ("sky_w", C.c_int32), ("sky_h", C.c_int32), ("sky_frame", f32 * 9),
        ("sky_step_size", f32), ("sky_bc2_sqrt", f32),
        ("prior_depth", vp), ("prior_aux", vp),
        ("prior_w", C.c_int32), ("prior_h", C.c_int32), ("has_depth", C.c_int32), ("has_sky_mask", C.c_int32),
        ("depth_weight", f32), ("sky_weight", f32), ("fill_weight", f32), ("huber_delta", f32), ("min_alpha", f32),
        ("mask_photometric", C.c_int32), ("loss_terms", vp),
        ("exposure", C.c_int32), ("cam_index", C.c_int32),
        ("expo_params", vp), ("expo_exp_avg", vp), ("expo_exp_avg_sq", vp), ("expo_grad", vp),
        ("expo_step_size", f32), ("expo_bc2_sqrt", f32), ("expo_reg", f32),
        ("log_max_scale_ratio", f32), ("expo_num_cams", C.c_int32),
    ]


_SIGS["msplat_cuda_set_prior"] = (i32, [vp, C.POINTER(Prior)])
_SIGS["msplat_cuda_render_aux_outputs"] = (i32, [vp, PP, PP])

# entry points added later in the build; bound when the library exports them
_OPTIONAL_SIGS: dict = {}


def lib():
    """The loaded library (built in-tree by msplat_street_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MsplatCudaError(
                f"{LIB_PATH} is missing: build it with `python -m msplat_street_b200.build` (needs nvcc)")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in {**_SIGS, **_OPTIONAL_SIGS}.items():
            fn = getattr(l, name, None)
            if fn is None:
                if name in _SIGS:
                    raise MsplatCudaError(f"{LIB_PATH} does not export {name}")
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().msplat_cuda_last_error().decode(errors="replace")
        raise _STATUS.get(status, MsplatCudaError)(f"msplat_cuda error {status}: {msg}")


def register(name: str, restype, argtypes) -> None:
    """Declare a signature for an optional entry point (bound on first load)."""
    _OPTIONAL_SIGS[name] = (restype, argtypes)
    if _lib is not None:
        fn = getattr(_lib, name, None)
        if fn is not None:
            fn.restype = restype
            fn.argtypes = argtypes
