"""Training loop host logic: the reference's Model and GaussianTrainer for this backend.

Restates core/src/model.cpp's training-side host code over the C-ABI:
 * capacity-backed parameter and Adam buffers with views of the active rows
   (setupOptimizers / refreshViews / ensureCapacity, model.cpp:81-193);
 * per-group learning rates and the log-linear means decay (model.cpp:100, :140-143),
   in float32 with the C library's logf / expf as the reference evaluates it;
 * Adam bias correction per step (fullIteration, :638-651);
 * the densification schedule (afterTrain, :199-245): every refine_every steps after
   the warm-up, densify while step < iterations / 2 and the reset-interval rule holds,
   reset opacities on the reset interval, clear the statistics (after_train_plan);
 * the resolution schedule: step s trains at downscale 2^max(num_downscales -
   s // resolution_schedule, 0) (image_sizing.cpp:129-133) on the target's area-
   downsampled pyramid level (Camera::getGPUImage, input_data.cpp:56-69);
 * SH degree ramp degrees_to_use = min(step // sh_degree_interval, sh_degree) (:535).
Steps are numbered from 1 as GaussianTrainer::step numbers them
(python/bindings.cpp:261-274): step s prepares its camera, trains, decays the means
learning rate and runs the densification schedule, all with s.
The camera set-up (prepareCam) is msplat_street_b200.camera.prepare_cam. The public
surface mirrors the reference's TrainingConfig / TrainingStats / GaussianTrainer
(python/msplat/_core.pyi:157-267) for in-memory datasets. Prior-guided training
(depth / sky / mask priors, learned sky, exposure, needle cap) follows
Model::configurePriors and the per-step PriorStep (model.cpp:548-625, 811-858), with
the prior maps built by msplat_street_b200.priors.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np
import torch

from . import formats
from . import priors as _priors
from .backend import AdamState, Context, GaussianParams, PriorStep
from .camera import CameraSetup, expf, logf, powf, prepare_cam, schedule_downscale_factor

LR_INIT = (0.00016, 0.005, 0.001, 0.0025, 0.000125, 0.05)  # model.cpp:100
MEANS_LR_FINAL = 0.0000016                                   # model.cpp:111
RESET_LOGIT = -1.3862943611198906                            # logit(0.2), model.cpp:236


@dataclass
class TrainingConfig:
    """Field names and defaults of the reference's TrainingConfig (python/bindings.cpp:27-60)."""

    iterations: int = 30000
    sh_degree: int = 3
    sh_degree_interval: int = 1000
    ssim_weight: float = 0.2
    num_downscales: int = 2
    resolution_schedule: int = 3000
    refine_every: int = 100
    warmup_length: int = 500
    reset_alpha_every: int = 30
    densify_grad_thresh: float = 0.0002
    densify_size_thresh: float = 0.01
    stop_screen_size_at: int = 4000
    split_screen_size: float = 0.05
    bg_color: Sequence[float] = (0.6130, 0.0101, 0.3984)
    # the thresholds Model::afterTrain hard-codes (model.cpp:218), exposed here
    cull_alpha_thresh: float = 0.1
    cull_scale_thresh: float = 0.5
    cull_screen_size: float = 0.15
    # learning rates (model.cpp:100); None keeps the reference's
    lrs: Optional[Sequence[float]] = None
    seed: int = 42


@dataclass
class TrainingStats:
    iteration: int
    splat_count: int
    ms_per_step: float


def sh_degrees_to_use(step: int, cfg: TrainingConfig) -> int:
    """Model::prepareCam's degreesToUse = min(step / shDegreeInterval, shDegree)
    (core/src/model.cpp:535)."""
    return min(step // max(cfg.sh_degree_interval, 1), cfg.sh_degree)


def means_lr(step: int, iterations: int) -> float:
    """Model::schedulersStep (core/src/model.cpp:140-143): the means learning rate after
    step ``step``, log-linear from 1.6e-4 to 1.6e-6 over the run, in float32 with the C
    library's logf / expf (the reference's std::log / std::exp on floats)."""
    f = np.float32
    t = min(max(f(step) / f(max(iterations, 1)), f(0.0)), f(1.0))
    return float(expf(logf(f(LR_INIT[0])) * (f(1.0) - t) + logf(f(MEANS_LR_FINAL)) * t))


@dataclass
class AfterTrainPlan:
    """What Model::afterTrain (core/src/model.cpp:199-245) does after step ``step``:
    densify (with these arguments) and / or reset opacities; the statistics are cleared
    whenever a plan exists."""

    step: int
    densify: bool
    reset: bool
    check_screen: bool
    check_huge: bool
    half_max_dim: float
    seed: int


def after_train_plan(step: int, cfg: TrainingConfig, num_cameras: int, last_width: int,
                     last_height: int) -> Optional[AfterTrainPlan]:
    """None on steps that are not refinement steps (step % refine_every != 0 or within
    the warm-up); else the plan. ``last_width`` / ``last_height``: the size the step
    trained at (its resolution-schedule level), as Model::lastWidth / lastHeight."""
    if not (step % cfg.refine_every == 0 and step > cfg.warmup_length):
        return None
    reset_interval = cfg.reset_alpha_every * cfg.refine_every
    stop_split_at = cfg.iterations // 2
    return AfterTrainPlan(
        step=step,
        densify=step < stop_split_at and step % reset_interval > num_cameras + cfg.refine_every,
        reset=step < stop_split_at and step % reset_interval == cfg.refine_every,
        check_screen=step < cfg.stop_screen_size_at,
        check_huge=step > cfg.refine_every * cfg.reset_alpha_every,
        half_max_dim=float(np.float32(0.5) * np.float32(max(last_width, last_height))),
        seed=(step * 2654435761) & 0xFFFFFFFF)


@dataclass
class View:
    """One training camera: its pose, intrinsics and target image."""

    cam_to_world: np.ndarray
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    image: Optional[np.ndarray] = None  # (H, W, 3) float32 in [0, 1]
    setup: CameraSetup = field(init=False)

    def __post_init__(self):
        self.setup = prepare_cam(self.cam_to_world, self.width, self.height, self.fx, self.fy, self.cx, self.cy)
        self._levels = {1: self.setup}

    def setup_at(self, factor: int) -> CameraSetup:
        """The camera at a resolution-schedule level (Model::prepareCam at downscale
        ``factor``)."""
        s = self._levels.get(factor)
        if s is None:
            s = prepare_cam(self.cam_to_world, self.width, self.height, self.fx, self.fy, self.cx, self.cy, factor)
            self._levels[factor] = s
        return s


class Dataset:
    """In-memory training set: views (pose + intrinsics + image) and a point cloud."""

    def __init__(self, views: List[View], points: np.ndarray, colors: np.ndarray):
        self.views = views
        self.points = np.ascontiguousarray(points, np.float32)
        self.colors = np.ascontiguousarray(colors, np.uint8)

    @classmethod
    def from_setups(cls, setups: List[CameraSetup], images, points, colors, poses) -> "Dataset":
        views = [View(p, s.width, s.height, s.fx, s.fy, s.cx, s.cy, img) for s, p, img in zip(setups, poses, images)]
        return cls(views, points, colors)


class GaussianTrainer:
    """3D Gaussian Splatting trainer on the B200 backend (reference: GaussianTrainer,
    python/bindings.cpp:217-427).

    ``views_per_step`` > 1 (or ``batched``) trains that many views per step with the
    batched step (msplat_cuda_train_batch: gradients summed over the views, one Adam
    step); ``graph`` replays a captured CUDA graph of that step."""

    def __init__(self, dataset: Dataset, config: TrainingConfig, init: Optional[GaussianParams] = None,
                 context: Optional[Context] = None, device: str = "cuda", views_per_step: int = 1,
                 batched: bool = False, graph: bool = False):
        self.cfg = config
        self.ds = dataset
        self.ctx = context or Context()
        self.device = device
        self.views_per_step = max(1, int(views_per_step))
        self.batched = batched or self.views_per_step > 1 or graph
        if graph:
            self.ctx.set_graph(True)
        if init is None:
            pts = torch.from_numpy(dataset.points).to(device)
            init = self.ctx.init_gaussians(pts, torch.from_numpy(dataset.colors), seed=42,
                                           opacity_logit=float(logf(np.float32(0.1) / np.float32(0.9))),
                                           sh_degree=config.sh_degree)
        self.lrs = list(config.lrs) if config.lrs is not None else list(LR_INIT)
        self._setup_buffers(init)
        self.current_step = 0
        self.adam_step = 0
        self.bg = np.asarray(config.bg_color, np.float32)
        self._targets = [torch.from_numpy(np.ascontiguousarray(v.image, np.float32)).to(device)
                         if v.image is not None else None for v in dataset.views]
        self._order: List[int] = []
        self._rng = np.random.default_rng(config.seed)
        self.stats = None
        self.last_loss = None
        self.radii_ready = False
        # the size the last step trained at (Model::lastWidth / lastHeight)
        self.last_width = dataset.views[0].width if dataset.views else 1
        self.last_height = dataset.views[0].height if dataset.views else 1
        self.last_views: List[int] = []  # the views the last step trained on
        # prior-guided training (configure_priors)
        self.prior_opts: Optional[_priors.PriorOptions] = None
        self.cam_priors: List[Optional[_priors.CameraPrior]] = [None] * len(dataset.views)
        self._prior_maps: List[Optional[tuple]] = [None] * len(dataset.views)
        self.sky: Optional[dict] = None
        self.exposure: Optional[dict] = None
        self.prior_loss_terms: Optional[torch.Tensor] = None

    # -- targets and their resolution-schedule levels ---------------------------------
    @property
    def _targets(self) -> List[Optional[torch.Tensor]]:
        return self._full_targets

    @_targets.setter
    def _targets(self, targets) -> None:
        self._full_targets = list(targets)
        self._pyramid = {}

    def target_at(self, ci: int, factor: int) -> Optional[torch.Tensor]:
        """View ci's target at downscale ``factor``: the full image area-downsampled to
        the level's size on the GPU and kept (Camera::getGPUImage, input_data.cpp:56-69)."""
        full = self._full_targets[ci]
        if full is None or factor <= 1:
            return full
        key = (ci, factor)
        t = self._pyramid.get(key)
        if t is None:
            s = self.ds.views[ci].setup_at(factor)
            t = self.ctx.resize_area(full, s.width, s.height)
            self._pyramid[key] = t
        return t

    def downscale_factor(self, step: int) -> int:
        """Model::getDownscaleFactor (model.cpp:195-197)."""
        return schedule_downscale_factor(step, self.cfg.num_downscales, self.cfg.resolution_schedule)

    # -- capacity buffers (model.cpp:81-193) ------------------------------------------
    def _setup_buffers(self, p: GaussianParams):
        n = p.n
        self.cap = max(4 * n, 4)
        self.num_active = n
        self.buf = []
        for t in p.tensors():
            shape = (self.cap,) + tuple(t.shape[1:])
            b = torch.zeros(shape, dtype=torch.float32, device=self.device)
            b[:n] = t
            self.buf.append(b)
        self.m1 = [torch.zeros_like(b) for b in self.buf]
        self.m2 = [torch.zeros_like(b) for b in self.buf]

    def ensure_capacity(self, needed: int) -> None:
        if needed <= self.cap:
            return
        new_cap = max(needed, 2 * self.cap)
        n = self.num_active

        def grow(b):
            nb = torch.zeros((new_cap,) + tuple(b.shape[1:]), dtype=b.dtype, device=b.device)
            nb[:n] = b[:n]
            return nb

        self.buf = [grow(b) for b in self.buf]
        self.m1 = [grow(b) for b in self.m1]
        self.m2 = [grow(b) for b in self.m2]
        self.cap = new_cap

    @property
    def params(self) -> GaussianParams:
        n = self.num_active
        return GaussianParams(*[b[:n] for b in self.buf])

    def _adam_view(self) -> AdamState:
        n = self.num_active
        st = AdamState([b[:n] for b in self.m1], [b[:n] for b in self.m2], self.lrs)
        st.step = self.adam_step
        return st

    # -- schedule -------------------------------------------------------------------
    def _next_camera(self) -> int:
        if not self._order:
            self._order = list(self._rng.permutation(len(self.ds.views)))
        return int(self._order.pop())

    def degrees_to_use(self, step: Optional[int] = None) -> int:
        """SH degrees used at ``step`` (default: the last step taken)."""
        return sh_degrees_to_use(self.current_step if step is None else step, self.cfg)

    def _schedulers_step(self, step: int) -> None:
        """Log-linear means LR decay (model.cpp:140-143)."""
        self.lrs[0] = means_lr(step, self.cfg.iterations)

    def _after_train(self, step: int) -> None:
        """Model::afterTrain (model.cpp:199-245)."""
        c = self.cfg
        plan = after_train_plan(step, c, len(self.ds.views), self.last_width, self.last_height)
        if plan is None:
            return
        if plan.densify and self.stats is not None:
            # a Gaussian may be both split and cloned: up to 4 N rows (the reference
            # reserves 3 N, model.cpp:158-193)
            self.ensure_capacity(4 * self.num_active)
            gn, vc, ms = self.stats[1], self.stats[0], self.stats[2]
            self.num_active = self.ctx.densify(
                self.num_active, self.buf, self.m1, self.m2, gn, vc, ms, plan.half_max_dim, plan.seed,
                grad_thresh=c.densify_grad_thresh, size_thresh=c.densify_size_thresh,
                screen_thresh=c.split_screen_size, check_screen=plan.check_screen, cull_alpha=c.cull_alpha_thresh,
                cull_scale=c.cull_scale_thresh, cull_screen=c.cull_screen_size, check_huge=plan.check_huge)
        if plan.reset:
            n = self.num_active
            self.ctx.opacity_reset(self.buf[5][:n], self.m1[5][:n], self.m2[5][:n], n, RESET_LOGIT)
        self.stats = None

    # -- prior-guided training (model.cpp:548-625, 811-858) ------------------------------
    def configure_priors(self, opts: "_priors.PriorOptions",
                         cam_priors: Optional[Sequence[Optional["_priors.CameraPrior"]]] = None) -> None:
        """Model::configurePriors: per-camera prior maps (CameraPrior, e.g. from
        priors.load_camera_prior; None where a camera has none), the learned sky's
        frame and initial texture, per-camera exposure at identity, the loss terms."""
        if self.batched and opts.active():
            raise ValueError("prior-guided training runs one view per step (views_per_step = 1, no graph)")
        self.prior_opts = opts
        n = len(self.ds.views)
        cps = list(cam_priors) if cam_priors is not None else [None] * n
        if len(cps) != n:
            raise ValueError(f"{len(cps)} camera priors for {n} views")
        self.cam_priors = cps if opts.wants_prior_files() else [None] * n
        self._prior_maps = [None if cp is None else
                            (torch.from_numpy(np.ascontiguousarray(cp.depth, np.float32)).to(self.device),
                             torch.from_numpy(np.ascontiguousarray(cp.aux, np.uint8)).to(self.device))
                            for cp in self.cam_priors]
        self.sky = None
        if opts.learn_sky:
            if opts.sky_width < 4 or opts.sky_height < 2:
                raise ValueError("sky texture must be at least 4x2")
            frame = _priors.compute_sky_frame([v.cam_to_world for v in self.ds.views])
            tex = _priors.init_sky_texture(self.ds.views, self.cam_priors, frame, opts.sky_width, opts.sky_height)
            t = torch.from_numpy(tex).to(self.device)
            self.sky = {"frame": frame, "steps": 0, "tex": t, "grad": torch.zeros_like(t),
                        "exp_avg": torch.zeros_like(t), "exp_avg_sq": torch.zeros_like(t)}
        self.exposure = None
        if opts.exposure and n:
            params = torch.zeros((n, 12), dtype=torch.float32, device=self.device)
            params[:, 0] = params[:, 4] = params[:, 8] = 1.0
            self.exposure = {"params": params, "exp_avg": torch.zeros_like(params),
                             "exp_avg_sq": torch.zeros_like(params),
                             "grad": torch.zeros(12, dtype=torch.float32, device=self.device), "steps": [0] * n}
        self.prior_loss_terms = torch.zeros(4, dtype=torch.float32, device=self.device)

    def _priors_active(self) -> bool:
        return self.prior_opts is not None and self.prior_opts.active()

    def _render_prior(self, force_aux: bool = False) -> Optional[PriorStep]:
        """renderPriorStep (model.cpp:549-561): the learned sky, or aux for depth renders."""
        ps = PriorStep(aux=force_aux)
        if self.prior_opts is not None and self.prior_opts.learn_sky and self.sky is not None:
            ps.aux = ps.sky = True
            ps.sky_tex = self.sky["tex"]
            ps.sky_frame = tuple(float(x) for x in self.sky["frame"])
        return ps if ps.aux else None

    def _train_prior(self, ci: int, step: int, adam: AdamState) -> PriorStep:
        """trainPriorStep (model.cpp:576-625) for camera ci at training step ``step``;
        advances the sky's and the camera's exposure Adam step counts."""
        o = self.prior_opts
        f = np.float32
        ps = self._render_prior(False) or PriorStep()
        cp, maps = self.cam_priors[ci], self._prior_maps[ci]
        depth_w = _priors.depth_weight_at(o, step, self.cfg.iterations) if cp is not None and cp.has_depth else 0.0
        sky_terms = cp is not None and cp.has_sky and (o.sky_alpha_weight > 0 or o.fill_weight > 0)
        masks = cp is not None and cp.has_mask and o.use_masks
        ps.aux = ps.aux or depth_w > 0 or sky_terms or masks

        def bias(lr, t):
            # std::pow(float, float) is the C library's powf (model.cpp:591-592, :618-619)
            return float(f(lr) / (f(1) - powf(adam.beta1, f(t)))), float(np.sqrt(f(1) - powf(adam.beta2, f(t))))

        if ps.sky:
            self.sky["steps"] += 1
            ps.sky_grad, ps.sky_exp_avg, ps.sky_exp_avg_sq = self.sky["grad"], self.sky["exp_avg"], self.sky[
                "exp_avg_sq"]
            ps.sky_step_size, ps.sky_bc2_sqrt = bias(o.sky_lr, self.sky["steps"])
        if cp is not None:
            ps.prior_depth, ps.prior_aux = maps
            ps.has_depth, ps.has_sky_mask = cp.has_depth, cp.has_sky
        ps.depth_weight = depth_w
        ps.sky_weight = o.sky_alpha_weight
        ps.fill_weight = o.fill_weight
        ps.huber_delta = o.depth_huber_delta
        ps.min_alpha = o.depth_min_alpha
        ps.mask_photometric = o.use_masks
        ps.loss_terms = self.prior_loss_terms
        if o.exposure and self.exposure is not None and 0 <= ci < len(self.exposure["steps"]):
            self.exposure["steps"][ci] += 1
            ps.exposure = True
            ps.cam_index = ci
            e = self.exposure
            ps.expo_params, ps.expo_exp_avg, ps.expo_exp_avg_sq, ps.expo_grad = (e["params"], e["exp_avg"],
                                                                                 e["exp_avg_sq"], e["grad"])
            ps.expo_step_size, ps.expo_bc2_sqrt = bias(o.exposure_lr, e["steps"][ci])
            ps.expo_reg = o.exposure_reg
        if o.max_scale_ratio > 1.0:
            ps.log_max_scale_ratio = float(logf(o.max_scale_ratio))
        return ps

    def prior_losses(self) -> dict:
        """Mean prior losses of the last step (GaussianTrainer::prior_losses,
        python/bindings.cpp:402-406). Synchronises."""
        if self.prior_loss_terms is None:
            return {"depth": 0.0, "sky": 0.0, "fill": 0.0}
        t = self.prior_loss_terms.cpu().numpy()
        return {"depth": float(t[0]), "sky": float(t[1]), "fill": float(t[2])}

    def render_depth(self, cam_idx: int):
        """Expected depth (dataset units) and alpha of a training camera
        (Model::renderDepth, model.cpp:860-877): an aux render, then
        msplat_finalize_depth. Returns two (H, W) float32 arrays."""
        v = self.ds.views[cam_idx]
        self.ctx.set_prior(self._render_prior(True))
        self.ctx.render(self.params, v.setup, self.bg, degrees_to_use=self.degrees_to_use())
        d, t = self.ctx.render_aux_outputs()
        depth, alpha = self.ctx.finalize_depth(d, t, 1.0 / self.crs_scale)
        return (depth.reshape(v.height, v.width).cpu().numpy(), alpha.reshape(v.height, v.width).cpu().numpy())

    def save_sky(self, path: str) -> None:
        """The learned sky texture as an 8-bit image (Model::saveSky, model.cpp:887-896)."""
        if self.sky is None:
            raise RuntimeError("No learned sky (enable learn_sky)")
        from PIL import Image
        tex = self.sky["tex"].cpu().numpy()
        Image.fromarray(np.clip(tex * np.float32(255.0), 0.0, 255.0).astype(np.uint8)).save(path)

    # -- public API -----------------------------------------------------------------
    def step(self, sync_loss: bool = False, target: Optional[torch.Tensor] = None) -> TrainingStats:
        """One training iteration (GaussianTrainer::step, python/bindings.cpp:261-284)."""
        t0 = time.perf_counter()
        step = self.current_step + 1  # GaussianTrainer::step numbers steps from 1
        factor = self.downscale_factor(step)
        dtu = self.degrees_to_use(step)
        n = self.num_active
        if self.stats is None:
            self.stats = tuple(torch.zeros(n, dtype=torch.float32, device=self.device) for _ in range(3))
        adam = self._adam_view()
        if self.batched:
            if target is not None:
                raise ValueError("a batched step takes its targets from the dataset")
            if self._priors_active():
                raise ValueError("prior-guided training runs one view per step")
            self.ctx.set_prior(None)
            views, picked = [], []
            for _ in range(self.views_per_step):
                ci = self._next_camera()
                picked.append(ci)
                gt = self.target_at(ci, factor)
                if gt is None:
                    raise ValueError(f"view {ci} has no target image")
                views.append((self.ds.views[ci].setup_at(factor), gt))
            losses = self.ctx.train_batch(self.params, adam, views, self.bg, self.stats,
                                          ssim_weight=self.cfg.ssim_weight, degrees_to_use=dtu, sync_loss=sync_loss)
            self.last_loss = float(np.mean(losses)) if losses is not None else None
            last = views[-1][0]
        else:
            ci = self._next_camera()
            picked = [ci]
            last = self.ds.views[ci].setup_at(factor)
            gt = target if target is not None else self.target_at(ci, factor)
            if gt is None:
                raise ValueError(f"view {ci} has no target image")
            self.ctx.set_prior(self._train_prior(ci, step, adam) if self._priors_active() else None)
            self.last_loss = self.ctx.train_step(self.params, adam, last, self.bg, gt, self.stats,
                                                 ssim_weight=self.cfg.ssim_weight, degrees_to_use=dtu,
                                                 sync_loss=sync_loss)
        self.last_width, self.last_height = last.width, last.height
        self.last_views = picked
        self.adam_step = adam.step
        self.current_step = step
        self._schedulers_step(step)
        self._after_train(step)
        return TrainingStats(step, self.num_active, (time.perf_counter() - t0) * 1e3)

    def train(self, callback: Optional[Callable[[TrainingStats], None]] = None, callback_every: int = 100) -> None:
        while self.current_step < self.cfg.iterations:
            st = self.step()
            if callback is not None and st.iteration % callback_every == 0:
                callback(st)

    def render_tensor(self, setup: CameraSetup) -> torch.Tensor:
        self.ctx.set_prior(self._render_prior(False))
        return self.ctx.render(self.params, setup, self.bg, degrees_to_use=self.degrees_to_use())

    def render(self, cam_idx: int) -> np.ndarray:
        """(H, W, 3) float32 render of a training camera."""
        return self.render_tensor(self.ds.views[cam_idx].setup).cpu().numpy()

    def render_from_pose(self, cam_to_world: np.ndarray, ref_cam_idx: int = 0) -> np.ndarray:
        """Render an OpenGL camera-to-world pose with a training camera's intrinsics."""
        v = self.ds.views[ref_cam_idx]
        setup = prepare_cam(np.asarray(cam_to_world, np.float32), v.width, v.height, v.fx, v.fy, v.cx, v.cy)
        return self.render_tensor(setup).cpu().numpy()

    def render_rgba8(self, cam_idx: int) -> np.ndarray:
        """(H, W, 4) uint8 render of a training camera (msplat_pack_rgba8's packing)."""
        return self.ctx.pack_rgba8(self.render_tensor(self.ds.views[cam_idx].setup))

    # -- files (python/bindings.cpp:372-386; core/src/model.cpp:256-496) ---------------
    crs_scale: float = 1.0
    crs_translation = (0.0, 0.0, 0.0)
    keep_crs: bool = False

    def export_ply(self, path: str) -> None:
        formats.save_ply(path, self.params.numpy(), self.current_step, self.crs_scale, self.crs_translation,
                         self.keep_crs)

    def export_splat(self, path: str) -> None:
        formats.save_splat(path, self.params.numpy(), self.crs_scale, self.crs_translation, self.keep_crs)

    def save_checkpoint(self, path: str) -> None:
        n = self.num_active
        ck = formats.Checkpoint(self.current_step, self.cfg.sh_degree, self.adam_step,
                                np.asarray(self.lrs, np.float32), LR_INIT[0], MEANS_LR_FINAL, self.params.numpy(),
                                [b[:n].cpu().numpy() for b in self.m1], [b[:n].cpu().numpy() for b in self.m2])
        if self.sky is not None:
            ck.sky = {"frame": self.sky["frame"], "steps": self.sky["steps"], "tex": self.sky["tex"].cpu().numpy(),
                      "exp_avg": self.sky["exp_avg"].cpu().numpy(),
                      "exp_avg_sq": self.sky["exp_avg_sq"].cpu().numpy()}
        if self.exposure is not None:
            e = self.exposure
            ck.exposure = {"params": e["params"].cpu().numpy(), "exp_avg": e["exp_avg"].cpu().numpy(),
                           "exp_avg_sq": e["exp_avg_sq"].cpu().numpy(), "steps": np.asarray(e["steps"], np.int32)}
        formats.save_checkpoint(path, ck)

    def load_checkpoint(self, path: str) -> int:
        """Restores parameters, Adam state, learning rates and the step; returns the
        step. Capacity becomes 4 N as Model::loadCheckpoint sets it (model.cpp:445-447)."""
        ck = formats.load_checkpoint(path)
        self._setup_buffers(GaussianParams(*[torch.from_numpy(a).to(self.device) for a in ck.params]))
        for g in range(6):
            self.m1[g][:ck.num_active] = torch.from_numpy(ck.exp_avg[g]).to(self.device).reshape(
                self.m1[g][:ck.num_active].shape)
            self.m2[g][:ck.num_active] = torch.from_numpy(ck.exp_avg_sq[g]).to(self.device).reshape(
                self.m2[g][:ck.num_active].shape)
        self.lrs = [float(x) for x in ck.lrs]
        self.adam_step = ck.adam_step
        self.current_step = ck.step
        self.stats = None
        # the learned sky and exposure are adopted only when this trainer uses them with
        # the same shapes (Model::loadCheckpoint, model.cpp:409-441)
        if ck.sky is not None and self.sky is not None and ck.sky["tex"].shape == tuple(self.sky["tex"].shape):
            for k in ("tex", "exp_avg", "exp_avg_sq"):
                self.sky[k].copy_(torch.from_numpy(np.ascontiguousarray(ck.sky[k])))
            self.sky["frame"] = np.asarray(ck.sky["frame"], np.float32).reshape(9)
            self.sky["steps"] = int(ck.sky["steps"])
        if (ck.exposure is not None and self.exposure is not None
                and ck.exposure["params"].shape == tuple(self.exposure["params"].shape)):
            for k in ("params", "exp_avg", "exp_avg_sq"):
                self.exposure[k].copy_(torch.from_numpy(np.ascontiguousarray(ck.exposure[k])))
            self.exposure["steps"] = [int(x) for x in ck.exposure["steps"]]
        return ck.step

    def evaluate(self, cam_idx: int):
        """(PSNR, SSIM, L1) of a training camera's render against its target
        (msplat_image_metrics)."""
        gt = self._targets[cam_idx]
        if gt is None:
            raise ValueError(f"view {cam_idx} has no target image")
        return self.ctx.image_metrics(self.render_tensor(self.ds.views[cam_idx].setup), gt)

    @property
    def splat_count(self) -> int:
        return self.num_active

    @property
    def iteration(self) -> int:
        return self.current_step
