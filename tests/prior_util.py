"""Seeded prior-guided inputs (core/metal/bindings.h:43-77, PriorStep) for parity tests.

``make_prior`` returns a dict of numpy arrays and scalars with the fields of the
oracle's orc_prior: a learned equirect sky, a depth prior at its own resolution with
invalid pixels and depth edges, a per-pixel aux map (confidence, sky, keep), an
affine exposure for several cameras and a needle cap. ``modes`` selects which of
them are on: "aux", "sky", "depth", "exposure", "needle".
"""
import numpy as np

ALL = ("aux", "sky", "depth", "exposure", "needle")


def make_prior(width, height, seed=0, modes=ALL, step=1, num_cams=3, cam_index=1, sky_w=32, sky_h=16,
               needle=0.7):
    rng = np.random.default_rng(seed)
    modes = set(modes)
    pr = {"aux": int("aux" in modes), "sky": int("sky" in modes), "exposure": int("exposure" in modes),
          "cam_index": cam_index, "log_max_scale_ratio": float(needle) if "needle" in modes else 0.0,
          "mask_photometric": 1, "huber_delta": 0.05, "min_alpha": 0.1,
          "depth_weight": 0.1, "sky_weight": 0.05, "fill_weight": 0.02}
    b1, b2 = 0.9, 0.999
    bc1 = np.float32(1.0 - b1 ** step)
    bc2s = np.float32(np.sqrt(np.float32(1.0 - b2 ** step)))
    if "sky" in modes:
        pr["sky_w"], pr["sky_h"] = sky_w, sky_h
        pr["sky_tex"] = rng.random((sky_h, sky_w, 3), dtype=np.float32)
        pr["sky_grad"] = np.zeros((sky_h, sky_w, 3), np.float32)
        pr["sky_exp_avg"] = (rng.standard_normal((sky_h, sky_w, 3)) * 1e-3).astype(np.float32)
        pr["sky_exp_avg_sq"] = (rng.random((sky_h, sky_w, 3)) * 1e-6).astype(np.float32)
        # a tilted orthonormal frame: up, azimuth 0, azimuth 90 degrees
        up = np.array([0.1, -0.95, 0.2]); up /= np.linalg.norm(up)
        e1 = np.cross(up, [0.0, 0.0, 1.0]); e1 /= np.linalg.norm(e1)
        e2 = np.cross(up, e1)
        pr["sky_frame"] = np.concatenate([up, e1, e2]).astype(np.float32)
        pr["sky_step_size"] = float(np.float32(1e-2) / bc1)
        pr["sky_bc2_sqrt"] = float(bc2s)
    if "depth" in modes:
        pw, ph = width // 2 + 3, height // 2 + 1
        coarse = 1.5 + 2.5 * rng.random(((ph + 3) // 4, (pw + 3) // 4)).astype(np.float32)
        d = np.kron(coarse, np.ones((4, 4), np.float32))[:ph, :pw]
        d = d * (1.0 + 0.01 * rng.standard_normal((ph, pw))).astype(np.float32)
        d[rng.random((ph, pw)) < 0.08] = 0.0
        aux = np.zeros((ph, pw, 4), np.uint8)
        aux[..., 0] = rng.integers(0, 256, (ph, pw))
        aux[..., 1] = np.where(rng.random((ph, pw)) < 0.2, 200, 30)
        aux[..., 2] = np.where(rng.random((ph, pw)) < 0.1, 0, 255)
        pr.update(prior_depth=np.ascontiguousarray(d, np.float32), prior_aux=aux, prior_w=pw, prior_h=ph,
                  has_depth=1, has_sky_mask=1)
    pr["loss_terms"] = np.zeros(4, np.float32)
    if "exposure" in modes:
        ident = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
        pr["expo_params"] = (ident + 0.05 * rng.standard_normal((num_cams, 12))).astype(np.float32)
        pr["expo_exp_avg"] = (rng.standard_normal((num_cams, 12)) * 1e-3).astype(np.float32)
        pr["expo_exp_avg_sq"] = (rng.random((num_cams, 12)) * 1e-6).astype(np.float32)
        pr["expo_grad"] = (rng.standard_normal(12) * 1e-3).astype(np.float32)
        pr["expo_step_size"] = float(np.float32(1e-3) / bc1)
        pr["expo_bc2_sqrt"] = float(bc2s)
        pr["expo_reg"] = 1e-2
    return pr


def restep(pr, step):
    """The per-step Adam scalars of ``pr`` for Adam step ``step`` (arrays kept)."""
    bc1 = np.float32(1.0 - 0.9 ** step)
    bc2s = float(np.float32(np.sqrt(np.float32(1.0 - 0.999 ** step))))
    if "sky_tex" in pr:
        pr["sky_step_size"], pr["sky_bc2_sqrt"] = float(np.float32(1e-2) / bc1), bc2s
    if "expo_params" in pr:
        pr["expo_step_size"], pr["expo_bc2_sqrt"] = float(np.float32(1e-3) / bc1), bc2s
    return pr


def copy_prior(pr):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in pr.items()}
