"""The training loop's host-side arithmetic against the reference's own Model (CPU).

The reference's core/src/model.cpp is compiled into oracle/_ref/libmsplat_ref_model.so
with its step's device work replaced by recording stubs (oracle/ref_model.cpp). Every
step of a run then yields, from the reference's own code, what its host side decides
and hands down, and each is compared with what this backend's trainer computes for
the same step, bit for bit:
  * prepareCam (model.cpp:498-546): level size, intrinsics, viewmat, projmat, camera
    position, SH degree and degrees_to_use, tile grid;
  * the resolution schedule (getDownscaleFactor, model.cpp:195-197);
  * fullIteration's Adam scalars (model.cpp:638-651) with the learning rates of that
    step, and the 1 / max(W, H) and 1 / (3 W H) scalars;
  * schedulersStep's means learning rate (model.cpp:140-143);
  * afterTrain (model.cpp:199-245): on which steps it densifies and resets opacities,
    and the densify arguments (thresholds, screen / huge checks, half the last
    training size, seed).
"""
import ctypes as C

import numpy as np
import pytest

from msplat_street_b200 import camera
from msplat_street_b200.backend import adam_step_scalars
from msplat_street_b200.camera import look_at, prepare_cam
from msplat_street_b200.trainer import (LR_INIT, RESET_LOGIT, TrainingConfig, after_train_plan, means_lr,
                                        sh_degrees_to_use)
from oracle_lib import PATHS, available

needs_ref = pytest.mark.skipif(not available("reference_model"), reason="reference Model code not built here")


def _P(a):
    return C.c_void_p(a.ctypes.data)


class RefModel:
    """The reference's Model over a small point cloud, driven one host-side step at a time."""

    def __init__(self, cfg: TrainingConfig, num_cameras: int, n_points: int = 48):
        self.lib = C.CDLL(PATHS["reference_model"])
        self.lib.ref_model_new.restype = C.c_void_p
        self.lib.ref_model_free.argtypes = [C.c_void_p]
        self.lib.ref_model_downscale_factor.argtypes = [C.c_void_p, C.c_int]
        rng = np.random.default_rng(7)
        xyz = rng.uniform(-1, 1, (n_points, 3)).astype(np.float32)
        rgb = rng.integers(0, 256, (n_points, 3), dtype=np.uint8)
        f = C.c_float
        self.m = self.lib.ref_model_new(
            n_points, _P(xyz), _P(rgb), num_cameras, cfg.num_downscales, cfg.resolution_schedule, cfg.sh_degree,
            cfg.sh_degree_interval, cfg.refine_every, cfg.warmup_length, cfg.reset_alpha_every,
            f(cfg.densify_grad_thresh), f(cfg.densify_size_thresh), cfg.stop_screen_size_at, f(cfg.split_screen_size),
            cfg.iterations)

    def close(self):
        self.lib.ref_model_free(C.c_void_p(self.m))

    def prepare_cam(self, c2w, w, h, intr, step):
        ints = np.zeros(6, np.int32)
        fl = np.zeros(4, np.float32)
        vm = np.zeros(16, np.float32)
        pm = np.zeros(16, np.float32)
        cp = np.zeros(3, np.float32)
        intr = np.asarray(intr, np.float32)
        c2w = np.ascontiguousarray(c2w, np.float32)
        self.lib.ref_model_prepare_cam(C.c_void_p(self.m), _P(c2w), w, h, _P(intr), step, _P(ints), _P(fl), _P(vm),
                                       _P(pm), _P(cp))
        return ints, fl, vm.reshape(4, 4), pm.reshape(4, 4), cp

    def iteration(self, c2w, w, h, intr, step):
        ss = np.zeros(6, np.float32)
        b2 = np.zeros(6, np.float32)
        fl = np.zeros(12, np.float32)
        it = np.zeros(10, np.int64)
        intr = np.asarray(intr, np.float32)
        c2w = np.ascontiguousarray(c2w, np.float32)
        self.lib.ref_model_iteration(C.c_void_p(self.m), _P(c2w), w, h, _P(intr), step, _P(ss), _P(b2), _P(fl),
                                     _P(it))
        return ss, b2, fl, it


def _cameras(n, seed=0):
    """Poses around the origin and intrinsics with odd sizes (the levels' integer
    division and per-axis ratios matter there)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        eye = rng.normal(size=3)
        eye = 3.0 * eye / np.linalg.norm(eye)
        w, h = int(rng.integers(97, 1999)), int(rng.integers(61, 1201))
        fx, fy = float(rng.uniform(0.4, 1.6) * w), float(rng.uniform(0.4, 1.6) * w)
        cx, cy = float(rng.uniform(0.3, 0.7) * w), float(rng.uniform(0.3, 0.7) * h)
        out.append((look_at(eye, rng.normal(size=3) * 0.2), w, h, (fx, fy, cx, cy)))
    return out


@needs_ref
@pytest.mark.parametrize("factor_steps", [(1, 2, 3, 2999, 3000, 5999, 6000, 6001, 30000)])
def test_prepare_cam_matches_reference(factor_steps):
    cfg = TrainingConfig()  # the reference's defaults: 2 downscales every 3000 steps
    ref = RefModel(cfg, 1)
    try:
        for c2w, w, h, intr in _cameras(40):
            for step in factor_steps:
                factor = camera.schedule_downscale_factor(step, cfg.num_downscales, cfg.resolution_schedule)
                ints, fl, vm, pm, cp = ref.prepare_cam(c2w, w, h, intr, step)
                s = prepare_cam(c2w, w, h, *intr, factor=factor)
                assert (s.width, s.height) == (ints[0], ints[1])
                assert (s.tiles_x, s.tiles_y) == (ints[4], ints[5])
                assert np.array_equal(np.float32([s.fx, s.fy, s.cx, s.cy]), fl)
                assert np.array_equal(s.viewmat, vm) and np.array_equal(s.projmat, pm)
                assert np.array_equal(s.cam_pos, cp)
                assert sh_degrees_to_use(step, cfg) == ints[3]
                assert ints[2] == 3  # SH degree 3 buffers
    finally:
        ref.close()


@needs_ref
def test_downscale_schedule_matches_reference():
    for nd, rs in ((2, 3000), (0, 3000), (3, 7), (1, 0), (31, 1)):
        cfg = TrainingConfig(num_downscales=nd, resolution_schedule=rs)
        ref = RefModel(cfg, 1)
        try:
            for step in list(range(0, 40)) + [2999, 3000, 3001, 5999, 6000, 9000, 10 ** 6]:
                assert camera.schedule_downscale_factor(step, nd, rs) == ref.lib.ref_model_downscale_factor(
                    C.c_void_p(ref.m), step), (nd, rs, step)
        finally:
            ref.close()


SCHEDULES = {
    # the reference's defaults over a short run: levels change, SH ramps, densify from 600
    "defaults_short": dict(iterations=4000, num_downscales=2, resolution_schedule=700, sh_degree_interval=500),
    # opacity resets inside the run (reset interval 300), refinement stops at iterations / 2
    "resets": dict(iterations=2600, num_downscales=1, resolution_schedule=900, reset_alpha_every=3,
                   refine_every=100, warmup_length=250, stop_screen_size_at=1000),
    # the street workload's schedule (full resolution, warm-up 400, 2000 steps)
    "street": dict(iterations=2000, num_downscales=0, refine_every=100, warmup_length=400, cull_alpha_thresh=0.005),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(SCHEDULES))
def test_training_schedule_matches_reference(name):
    cfg = TrainingConfig(**SCHEDULES[name])
    cams = _cameras(5, seed=3)
    ref = RefModel(cfg, len(cams))
    lrs = list(LR_INIT)
    last_w = last_h = 1
    densified = resets = 0
    try:
        for step in range(1, cfg.iterations + 1):
            c2w, w, h, intr = cams[(step * 7) % len(cams)]
            ss_ref, b2_ref, fl, it = ref.iteration(c2w, w, h, intr, step)
            factor = camera.schedule_downscale_factor(step, cfg.num_downscales, cfg.resolution_schedule)
            s = prepare_cam(c2w, w, h, *intr, factor=factor)
            assert (it[0], it[1]) == (s.width, s.height), step
            # Adam scalars of step `step` (Adam's own step count equals the training step)
            ss, b2 = adam_step_scalars(lrs, step)
            assert np.array_equal(ss, ss_ref) and np.array_equal(b2, b2_ref), step
            assert np.float32(1.0) / np.float32(max(s.width, s.height)) == fl[1]
            assert np.float32(1.0) / np.float32(s.width * s.height * 3) == fl[2]
            # schedulersStep
            lrs[0] = means_lr(step, cfg.iterations)
            assert np.float32(lrs[0]) == fl[0], step
            # afterTrain
            last_w, last_h = s.width, s.height
            plan = after_train_plan(step, cfg, len(cams), last_w, last_h)
            dens = plan is not None and plan.densify
            reset = plan is not None and plan.reset
            assert dens == bool(it[2]) and reset == bool(it[8]), step
            if dens:
                densified += 1
                want = np.float32([cfg.densify_grad_thresh, cfg.densify_size_thresh, cfg.split_screen_size,
                                   0.1, 0.5, 0.15, plan.half_max_dim])
                assert np.array_equal(want, fl[3:10]), step
                assert (int(plan.check_screen), int(plan.check_huge), plan.seed) == (it[5], it[6], it[7]), step
            if reset:
                resets += 1
                assert fl[10] == np.float32(RESET_LOGIT)
    finally:
        ref.close()
    # every schedule above densifies; "resets" also resets opacities
    assert densified > 0
    assert resets > 0 or name != "resets"
