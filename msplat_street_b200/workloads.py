"""Seeded training workloads shared by the benchmark and the tests.

street_plain(): the street-scale plain method -- a 500,000-Gaussian ground-truth
scene in a 20 x 4 x 20 m box, 16 target renders at 1024 x 512 from cameras on a
10 m line at 1.5 m height with +-30 degree yaw jitter, and a training start of
100,000 ground-truth means with N(0, 5 cm) jitter whose scales come from the exact
3-NN mean distance. Densify every 100 steps from step 500 (warm-up 400, so step 500
is the first refinement), split/clone above a view-space gradient of 2e-4, prune
below opacity 0.005; iterations 2000 (so refinement stops at step 1000, the
reference's iterations / 2 rule). Every step trains at the full 1024 x 512 (no
resolution schedule: num_downscales 0).
"""
from __future__ import annotations

import numpy as np
import torch

from . import scenes
from .backend import Context, GaussianParams
from .trainer import Dataset, GaussianTrainer, TrainingConfig

STREET_GT_N = 500_000
STREET_INIT_N = 100_000
STREET_W, STREET_H, STREET_F = 1024, 512, 512.0
STREET_VIEWS = 16
BACKGROUND = np.array([0.6130, 0.0101, 0.3984], np.float32)


def street_config(iterations: int = 2000) -> TrainingConfig:
    return TrainingConfig(iterations=iterations, sh_degree=3, sh_degree_interval=1000, ssim_weight=0.2,
                          num_downscales=0, refine_every=100, warmup_length=400, densify_grad_thresh=2e-4,
                          cull_alpha_thresh=0.005)


def street_views(gt_n: int = STREET_GT_N):
    gt = scenes.street_scene(0, gt_n)
    poses = scenes.street_camera_poses(STREET_VIEWS, seed=2)
    setups = scenes.street_cameras(STREET_W, STREET_H, STREET_F, STREET_VIEWS, seed=2)
    return gt, poses, setups


def street_plain(ctx: Context, gt_n: int = STREET_GT_N, init_n: int = STREET_INIT_N, iterations: int = 2000,
                 device: str = "cuda"):
    """(trainer, targets) for the street-scale plain config; targets rendered on the GPU."""
    gt, poses, setups = street_views(gt_n)
    pg = GaussianParams.from_numpy(gt, device)
    targets = [ctx.render(pg, s, BACKGROUND).clone() for s in setups]
    del pg
    pts, rgb = scenes.jittered_init_points(gt, init_n, seed=3)
    ds = Dataset.from_setups(setups, [None] * len(setups), pts, rgb, poses)
    tr = GaussianTrainer(ds, street_config(iterations), context=ctx, device=device)
    tr._targets = targets
    return tr, targets


# --- batching: the street scene and schedule, 16 cameras of mixed resolutions ---------

BATCH_RESOLUTIONS = ((640, 480), (1024, 512), (1280, 720), (1600, 1060))


def street_mixed_setups(seed: int = 4):
    """The 16 street poses, each at a resolution drawn uniformly (seeded) from
    BATCH_RESOLUTIONS, focal length half the width (the plain config's 90 degree
    horizontal field of view)."""
    from .camera import prepare_cam
    poses = scenes.street_camera_poses(STREET_VIEWS, seed=2)
    rng = np.random.default_rng(seed)
    out = []
    for p in poses:
        w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        out.append(prepare_cam(p, w, h, 0.5 * w, 0.5 * w, w / 2.0, h / 2.0))
    return poses, out


def street_batched(ctx: Context, views_per_step: int = 8, graph: bool = True, batched: bool = True,
                   gt_n: int = STREET_GT_N, init_n: int = STREET_INIT_N, iterations: int = 2000,
                   device: str = "cuda"):
    """(trainer, targets) for the batching config: street_plain's scene, start and
    schedule with the mixed-resolution cameras; ``views_per_step`` views per step
    through the batched step (``batched=False``: the plain per-view step)."""
    gt = scenes.street_scene(0, gt_n)
    poses, setups = street_mixed_setups()
    pg = GaussianParams.from_numpy(gt, device)
    targets = [ctx.render(pg, s, BACKGROUND).clone() for s in setups]
    del pg
    pts, rgb = scenes.jittered_init_points(gt, init_n, seed=3)
    ds = Dataset.from_setups(setups, [None] * len(setups), pts, rgb, poses)
    tr = GaussianTrainer(ds, street_config(iterations), context=ctx, device=device,
                         views_per_step=views_per_step if batched else 1, batched=batched,
                         graph=graph and batched)
    tr._targets = targets
    return tr, targets
