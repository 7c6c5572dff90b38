"""Benchmark: street-scale plain training, iterations per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (msplat_street_b200.workloads.street_plain): a 500,000-Gaussian ground-truth
street scene (20 x 4 x 20 m), 16 target views at 1024 x 512, training from 100,000
kNN-initialised Gaussians with the densification schedule of the 2,000-iteration
street config. A step is one training iteration of that schedule (one view): W
untimed warm-up iterations, then K timed ones that continue the schedule, with any
densification that falls in the window inside the timed step.

value: iterations/s with the targets resident in HBM, device-timed with CUDA events
per step (L2 flushed by a 256 MB write between steps, outside the events); e2e: the
same schedule replayed through the public API with each step's target copied from
pinned host memory (on a copy stream, one step ahead, overlapping the previous
step's kernels) and each step's loss read back into pinned memory (waited for once
the next step is queued), wall-clock timed. Training does not
shard without a gradient exchange, so N GPUs run N independent replicas ("replicas
only", weak scaling); value is the sum over ranks of K / max-over-ranks time.

--impl reference times the reference's own CPU backend (core/cpu, built into
oracle/_ref) on a bounded sample of the same schedule on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "train iters/s (street plain, 1024x512)"
UNIT = "iters/s"
WORKLOAD = ("street-plain: 500k-Gaussian GT scene (20x4x20 m), 16 views 1024x512, train from 100k kNN-init "
            "Gaussians, densify every 100 from step 500, 2000-iteration schedule")
HBM_FALLBACK_GBS = 6650.0


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms around the timed
    region. A timed region can be shorter than nvidia-smi's start-up, so entering waits
    (at most 5 s) for the first sample and leaving waits (at most 2 s) for one taken
    after the region ended: the record always brackets the region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            self._wait_rows(1, 5.0)
        except Exception:
            self.proc = None
        return self

    def _rows(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.count(",") >= 8)
        except Exception:
            return 0

    def _wait_rows(self, n: int, limit_s: float) -> None:
        t0 = time.perf_counter()
        while self.proc is not None and self.proc.poll() is None and self._rows() < n \
                and time.perf_counter() - t0 < limit_s:
            time.sleep(0.01)

    def __exit__(self, *exc):
        if self.proc is not None:
            self._wait_rows(self._rows() + 1, 2.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        util = [num(r[9]) for r in rows if len(r) > 9 and num(r[9]) is not None]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "gpu_util_pct": statistics.mean(util) if util else None}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ------------------------------------------------------------------------------------
# CPU baseline: the reference's own core/cpu backend on the host cores

def cpu_reference_run(seconds: float, max_steps: int, warmup: int = 1):
    """Trains the same street schedule with the reference's CPU backend until ``seconds``
    of timed work or ``max_steps`` iterations; returns (iters/s, steps, threads, n)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from msplat_street_b200 import scenes, workloads
    from oracle_lib import Oracle, available, new_adam_state
    kind = "reference_fast" if available("reference_fast") else "restatement"
    ref = Oracle(kind)
    gt, poses, setups = workloads.street_views(workloads.STREET_GT_N)
    pts, rgb = scenes.jittered_init_points(gt, workloads.STREET_INIT_N, seed=3)
    s, q, d, o = ref.init_gaussians(pts, rgb, 42, float(np.log(0.1 / 0.9)))
    g = scenes.Gaussians(pts.copy(), s, q, d, np.zeros((pts.shape[0], 15, 3), np.float32), o)
    lrs = [0.00016, 0.005, 0.001, 0.0025, 0.000125, 0.05]
    m1 = [np.zeros_like(a) for a in g.arrays()]
    m2 = [np.zeros_like(a) for a in g.arrays()]
    st = {k: np.zeros(g.n, np.float32) for k in ("vis", "gn", "ms")}
    order = list(np.random.default_rng(42).permutation(len(setups)))
    targets = {}
    done, elapsed, step = 0, 0.0, 0
    while done < max_steps and (elapsed < seconds or done == 0):
        ci = int(order[step % len(order)])
        if ci not in targets:
            targets[ci] = ref.render(gt, setups[ci], workloads.BACKGROUND)
        step += 1
        ad = new_adam_state(g, lrs, step)
        ad["m1"], ad["m2"] = m1, m2
        t0 = time.perf_counter()
        ref.train_step(g, setups[ci], workloads.BACKGROUND, targets[ci], ad, st,
                       degrees_to_use=min(step // 1000, 3))
        dt = time.perf_counter() - t0
        if step > warmup:
            elapsed += dt
            done += 1
    threads = int(os.environ.get("MSPLAT_THREADS", os.cpu_count() or 1)) if kind != "restatement" else \
        (os.cpu_count() or 1)
    return done / elapsed, done, threads, g.n, kind


def run_reference(args, world, rank):
    if rank != 0:
        return
    try:
        rate, done, threads, n, kind = cpu_reference_run(seconds=min(60.0, 6.0 * max(args.steps, 1)),
                                                         max_steps=max(args.steps, 1), warmup=min(args.warmup, 1))
    except Exception as e:  # the reference build is missing
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU backend not runnable: {e}"}))
        return
    sample = (f"{done} training iterations of the street schedule from step 2 ({n} Gaussians, 1024x512) with the "
              f"reference core/cpu backend, {threads} host threads")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1000.0 / rate, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "host threads"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads,
                             "kind": "reference" if kind.startswith("reference") else "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch
    from msplat_street_b200 import workloads
    from msplat_street_b200.backend import Context

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    total_steps = args.warmup + args.steps
    iters = max(2000, total_steps)

    # ---- device-timed pass: targets resident in HBM ----
    ctx = Context()
    if args.raster_shape is not None:
        ctx.set_raster_shape(args.raster_shape)
    trainer, targets = workloads.street_plain(ctx, iterations=iters)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    for _ in range(args.warmup):
        trainer.step()
    torch.cuda.synchronize()
    ctx.enable_stage_timing(True)
    ctx.drain_stage_times()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    n_isects, n_gauss = [], []
    pair_sum = torch.zeros(2, dtype=torch.int64, device=dev)
    window = {"first": trainer.iteration + 1, "sh_first": trainer.degrees_to_use(trainer.iteration + 1),
              "gaussians_first": trainer.splat_count, "densify": []}
    barrier(world, dev)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            flush.zero_()
            n_gauss.append(trainer.splat_count)
            evs[i][0].record()
            st = trainer.step()
            evs[i][1].record()
            n_isects.append(ctx.num_isects())  # known on the host since the step's binning
            ctx.add_pair_counts(pair_sum)  # outside the events: a counting kernel, no readback
            if st.splat_count != n_gauss[-1]:
                window["densify"].append(st.iteration)
        torch.cuda.synchronize()
    barrier(world, dev)
    pairs = [tuple(float(x) / args.steps for x in pair_sum.cpu().tolist())]  # per-step means
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), world, dev)
    stages = ctx.drain_stage_times()
    ctx.enable_stage_timing(False)
    final_n = trainer.splat_count
    value = world * args.steps / (total_ms / 1e3)
    window.update(last=trainer.iteration, sh_last=trainer.degrees_to_use(), gaussians_last=final_n)
    timed_window = (f"iterations {window['first']}..{window['last']} of the 2000-iteration schedule: SH degree "
                    f"{window['sh_first']}..{window['sh_last']}, {window['gaussians_first']}..{window['gaussians_last']}"
                    f" Gaussians, densify steps {window['densify'] or 'none'}")

    if args.quick:  # device pass only (profiling runs)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "quick": True,
                              "timed_window": timed_window,
                              "stages_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in stages.items()},
                              "isects_mean": float(np.mean(n_isects)),
                              "pairs_mean": [float(np.mean([p[0] for p in pairs])),
                                             float(np.mean([p[1] for p in pairs]))]}))
        return

    # ---- the rest of the schedule: 20-step windows spread over it (rank 0 times them
    # on the same trainer, densification steps included) ----
    sched = schedule_sample(trainer, ctx, flush, dev) if rank == 0 else None
    knn = knn_rate(trainer, ctx) if rank == 0 else None

    # ---- end-to-end pass through the public API: host targets, loss read back ----
    ctx2 = Context()
    if args.raster_shape is not None:
        ctx2.set_raster_shape(args.raster_shape)
    trainer2, targets2 = workloads.street_plain(ctx2, iterations=iters)
    host_targets = [t.cpu().pin_memory() for t in targets2]
    del targets2
    trainer2._targets = [None] * len(host_targets)
    prefetch = TargetPrefetch(trainer2, host_targets, dev)
    for _ in range(args.warmup):
        trainer2.step(target=prefetch.next(), sync_loss=True)
    # every step's loss is read back into pinned memory; the host waits for step i's
    # value after queueing step i + 1, so reading it does not leave the GPU idle
    loss_host = torch.zeros(2, dtype=torch.float32).pin_memory()
    losses = []
    barrier(world, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prev = None
    for i in range(args.steps):
        trainer2.step(target=prefetch.next())
        ev = ctx2.read_loss_async(loss_host[i % 2:i % 2 + 1])
        if prev is not None:
            prev[0].synchronize()
            losses.append(float(loss_host[prev[1]]))
        prev = (ev, i % 2)
    prev[0].synchronize()
    losses.append(float(loss_host[prev[1]]))
    torch.cuda.synchronize()
    assert len(losses) == args.steps and np.isfinite(losses).all(), "a step's loss was not read back"
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
    barrier(world, dev)
    e2e = world * args.steps / e2e_s
    h2d = int(host_targets[0].numel() * 4)

    # ---- roofline of the dominant stage (live CUDA-event durations) ----
    peaks, peak_kind = measured_peaks()
    ck = clocks.summary()
    roof = roofline(stages, n_isects, float(np.mean(n_gauss)), peaks, peak_kind, pairs, ck.get("sm_mhz"))
    thr = throughput(stages, n_isects, float(np.mean(n_gauss)), pairs, peaks, peak_kind, ck.get("sm_mhz"))
    if knn:
        thr["knn"] = knn

    # ---- differentiable path: recomputed vs stored transmittance (rank 0) ----
    diff = None
    if rank == 0:
        try:
            diff = differentiation_report(dev)
        except Exception as e:
            diff = {"error": str(e)}
    chunk = None
    if rank == 0:
        try:
            chunk = chunked_report(dev)
        except Exception as e:
            chunk = {"error": str(e)}

    # ---- render serving (rank 0) ----
    serve = None
    if rank == 0 and args.serving_seconds > 0:
        try:
            serve = serving_report(dev, args.serving_seconds)
        except Exception as e:
            serve = {"error": f"{type(e).__name__}: {e}"}

    # ---- batched multi-view training vs the plain per-view step (rank 0) ----
    batching = None
    if rank == 0 and not args.no_batching:
        try:
            batching = batching_report(dev)
        except Exception as e:
            batching = {"error": f"{type(e).__name__}: {e}"}

    # ---- the reference's C++ callers' path: bindings.h with host tensors (rank 0) ----
    bindings = None
    if rank == 0:
        try:
            bindings = bindings_report(dev)
        except Exception as e:
            bindings = {"error": f"{type(e).__name__}: {e}"}

    # ---- CPU baseline (rank 0, N=1 only) ----
    cpu = None
    if world == 1:
        try:
            rate, done, threads, n, kind = cpu_reference_run(seconds=15.0, max_steps=200)
            cpu = {"value": rate, "unit": UNIT, "cores": threads,
                   "kind": "reference" if kind.startswith("reference") else "port",
                   "sample": f"{done} iterations of the same schedule from step 2 ({n} Gaussians), "
                             f"reference core/cpu backend built -O3, all host threads"}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "timed_window": timed_window,
                       "gaussians_end": final_n, "isects_mean": float(np.mean(n_isects)),
                       "l2": "256 MB write between timed steps", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4},
            "gpu_launches": int(args.steps * launches_per_step(np.mean(n_isects), final_n)),
            "roofline": roof,
            "throughput": thr,
            "schedule_sample": sched,
            "stages_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in stages.items()},
            "clocks": {"sm_mhz": ck.get("sm_mhz"), "sm_max_mhz": ck.get("sm_max_mhz"), "reasons": ck.get("reasons")},
            "cpu_baseline": cpu,
            "differentiation": diff,
            "chunked_compositing": chunk,
            "serving": serve,
            "batching": batching,
            "bindings_h": bindings,
        }
        if serve and "rates" in serve:
            hi = serve["rates"].get("1000") or next(iter(serve["rates"].values()))
            line["render"] = {"p50_ms": hi["batched"]["p50_ms"], "p99_ms": hi["batched"]["p99_ms"],
                              "p99_1080p_ms": hi["batched"]["p99_1080p_ms"],
                              "plain_p50_ms": hi["plain"]["p50_ms"], "plain_p99_ms": hi["plain"]["p99_ms"],
                              "at_rate_req_s": 1000}
        print(json.dumps(line))


def bindings_report(dev, steps: int = 300, warmup: int = 10) -> dict:
    """Training-step throughput on the small plain config (10k Gaussians, 256x256)
    through bindings.h with host tensors -- the path core/src/model.cpp and the CLI take
    (msplat_street_b200/_build/train_bindings, wall clock, every call staging its
    tensors to the device and back) -- next to the same training from C++ straight
    through the C-ABI with device-resident tensors (the same binary, mode c_abi, wall
    clock) and through the Python API (CUDA events)."""
    import torch
    from msplat_street_b200 import build, scenes
    from msplat_street_b200.backend import AdamState, Context, GaussianParams
    from msplat_street_b200.trainer import LR_INIT
    out = {"config": "10k Gaussians, 256x256, SH degree 3, L1 + 0.2 SSIM, Adam"}
    for mode in ("bindings_h", "c_abi"):
        if os.path.exists(build.TRAIN_BINDINGS):
            r = subprocess.run([build.TRAIN_BINDINGS, str(steps), str(warmup), mode], capture_output=True, text=True,
                               timeout=300)
            line = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out[mode] = json.loads(line[-1]) if r.returncode == 0 and line else {"error": r.stderr[-300:]}
        else:
            out[mode] = {"error": "train_bindings not built (needs the reference headers at build time)"}
    ctx = Context()
    cam = scenes.small_camera()
    bg = np.array([0.6130, 0.0101, 0.3984], np.float32)
    gt = ctx.render(GaussianParams.from_numpy(scenes.small_scene(1)), cam, bg).clone()
    p = GaussianParams.from_numpy(scenes.small_scene(0))
    adam = AdamState.zeros_like(p, LR_INIT)
    stats = tuple(torch.zeros(p.n, device=dev) for _ in range(3))
    for _ in range(warmup):
        ctx.train_step(p, adam, cam, bg, gt, stats)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ctx.train_step(p, adam, cam, bg, gt, stats)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out["python_api"] = {"iters_per_s": 1e3 / ms, "ms_per_step": ms, "steps": steps}
    ctx.close()
    return out


def batching_report(dev, views: int = 480, warmup_views: int = 48, views_per_step: int = 8):
    """Mixed-resolution street training (16 cameras at 640x480 / 1024x512 / 1280x720 /
    1600x1060): the plain per-view step, the batched step (views_per_step views per
    step, one launch per stage) without and with CUDA-graph replay. Each arm trains
    ``views`` views after ``warmup_views`` from the same start (before the first
    densification), wall-clock timed between device synchronisations."""
    import torch
    from msplat_street_b200 import workloads
    from msplat_street_b200.backend import Context

    out = {"views_per_step": views_per_step, "views_timed": views,
           "resolutions": [list(r) for r in workloads.BATCH_RESOLUTIONS]}
    arms = (("plain", False, False), ("batched", True, False), ("batched_graph", True, True))
    for name, batched, graph in arms:
        ctx = Context()
        tr, _ = workloads.street_batched(ctx, views_per_step=views_per_step, graph=graph, batched=batched)
        per = views_per_step if batched else 1
        for _ in range(max(warmup_views // per, 3)):
            tr.step()
        tuned = None
        if graph:
            # the autotuner on this arm before it is timed: every compiled rasterizer
            # staging variant x batched-forward block shape (16x16, 16x8, 8x8) timed on
            # the graph-replayed step, interleaved over rounds; the step keeps the best
            from msplat_street_b200.autotune import tune_raster
            tuned = tune_raster([ctx], tr.step, warmup=1, reps=4, rounds=2, shapes=[0, 1, 2])
        torch.cuda.synchronize()
        steps = views // per
        if not graph:  # the eager arms report per-view device time by stage (CUDA events)
            ctx.enable_stage_timing(True)
            ctx.drain_stage_times()
        with ClockSampler(torch.cuda.current_device()) as smi:
            t0 = time.perf_counter()
            for _ in range(steps):
                tr.step()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        out[name] = {"views_per_s": steps * per / dt, "steps_per_s": steps / dt, "ms_per_step": dt / steps * 1e3,
                     "gaussians": tr.splat_count, "gpu_util_pct": smi.summary().get("gpu_util_pct")}
        if not graph:
            st = ctx.drain_stage_times()
            ctx.enable_stage_timing(False)
            out[name]["stage_ms_per_view"] = {k: a / max(c, 1) / per for k, (a, c) in st.items()}
            out[name]["device_ms_per_view"] = sum(out[name]["stage_ms_per_view"].values())
            out[name]["wall_ms_per_view"] = dt / (steps * per) * 1e3
        if graph:
            out[name]["graph"] = ctx.graph_stats()
            out[name]["autotune"] = {"best": tuned["best"], "best_staging": tuned["variants"][tuned["best"]],
                                     "best_shape": tuned["shapes"][tuned["best_shape"]],
                                     "ms_per_step_by_variant_shape": {str(k): v for k, v in tuned["ms"].items()}}
        del tr
        ctx.close()
        torch.cuda.empty_cache()
    for name in ("batched", "batched_graph"):
        out[name]["views_per_s_vs_plain"] = out[name]["views_per_s"] / out["plain"]["views_per_s"]
    out["small"] = small_batching_report(views_per_step)
    return out


def small_batching_report(views_per_step: int = 8, views: int = 960):
    """Where one view cannot fill the GPU: a 10 k-Gaussian scene (the small plain
    config's distributions), 16 cameras at 256 x 256 on a 3 m sphere (256 tiles each,
    fewer than the resident blocks of one wave). Plain per-view steps vs batched steps
    with graph replay; wall-clock views/s."""
    import torch
    from msplat_street_b200 import scenes
    from msplat_street_b200.backend import Context, GaussianParams
    from msplat_street_b200.trainer import Dataset, GaussianTrainer, TrainingConfig
    from msplat_street_b200.workloads import BACKGROUND

    from msplat_street_b200.camera import prepare_cam
    rng = np.random.default_rng(12)
    poses = [scenes.sphere_pose(rng, 3.0) for _ in range(16)]
    f = 0.5 * 256 / np.tan(np.radians(30.0))
    setups = [prepare_cam(p, 256, 256, f, f, 128.0, 128.0) for p in poses]
    gt = GaussianParams.from_numpy(scenes.small_scene(1))
    ctx0 = Context()
    targets = [ctx0.render(gt, s, BACKGROUND).clone() for s in setups]
    init = scenes.small_scene(0)
    out = {"scene": "10k Gaussians, 16 views 256x256"}
    for name, batched, graph in (("plain", False, False), ("batched_graph", True, True)):
        ctx = Context()
        ds = Dataset.from_setups(setups, [None] * 16, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.uint8),
                                 poses)
        # full resolution, no densification in the window
        cfg = TrainingConfig(iterations=100000, warmup_length=10 ** 9, num_downscales=0)
        tr = GaussianTrainer(ds, cfg, init=GaussianParams.from_numpy(init), context=ctx,
                             views_per_step=views_per_step if batched else 1, batched=batched, graph=graph)
        tr._targets = targets
        per = views_per_step if batched else 1
        for _ in range(max(32 // per, 3)):
            tr.step()
        tuned = None
        if graph:  # the same tuner as the street arm's, on this step
            from msplat_street_b200.autotune import tune_raster
            tuned = tune_raster([ctx], tr.step, warmup=1, reps=6, rounds=2, shapes=[0, 1, 2])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(views // per):
            tr.step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[name] = {"views_per_s": (views // per) * per / dt}
        if tuned:
            out[name]["autotune"] = {"best_staging": tuned["variants"][tuned["best"]],
                                     "best_shape": tuned["shapes"][tuned["best_shape"]]}
        ctx.close()
    out["batched_graph"]["views_per_s_vs_plain"] = out["batched_graph"]["views_per_s"] / out["plain"]["views_per_s"]
    return out


def serving_report(dev, seconds: float, rates=(200.0, 1000.0, 5000.0)):
    """Render serving: 32 resident scenes (Gaussian counts log-uniform in [5e4, 3e6],
    SH degree 3, FP32) under a 150 GB budget; Poisson request streams at each rate for
    ``seconds`` with random cameras on a 5 m sphere and resolutions uniform over
    {512x512, 1280x720, 1920x1080}. The batched server (3 slots, continuous batching
    into the persistent rasterizer) and serial plain single-view renders serve the same
    stream; latency = image complete on the device - arrival. "saturated" offers 1,500
    requests at once (closed-loop capacity)."""
    import torch
    from msplat_street_b200 import serving
    from msplat_street_b200.workloads import BACKGROUND

    sizes = serving.scene_sizes(32, 50_000, 3_000_000, seed=5)
    store = serving.SceneStore(150 * 10 ** 9, device=dev)
    for i, n in enumerate(sizes):
        store.add(i, serving.random_scene_tensors(n, 100 + i, device=dev), resident=True, host_copy=False)
    torch.cuda.synchronize()
    srv = serving.RenderServer(store, BACKGROUND, slots=3, max_batch=16, max_batch_pixels=16 * 1920 * 1080)
    plain = serving.RenderServer(store, BACKGROUND, mode="plain")
    warm = serving.poisson_requests(2000.0, 0.1, len(sizes), seed=1)
    srv.run(warm, realtime=False)
    plain.run(warm, realtime=False)
    out = {"scenes": len(sizes), "gaussians_total": int(sum(sizes)), "budget_gb": 150,
           "resident_gb": store.resident_bytes / 1e9, "stream_seconds": seconds, "rates": {}}
    for rate in rates:
        reqs = serving.poisson_requests(rate, seconds, len(sizes), seed=int(rate))
        b = serving.latency_summary(srv.run(reqs, realtime=True))
        p = serving.latency_summary(plain.run(reqs, realtime=True))
        out["rates"][str(int(rate))] = {"batched": b, "plain": p}
    burst = serving.poisson_requests(1e6, 1500 / 1e6, len(sizes), seed=3)
    out["saturated"] = {"requests": len(burst),
                        "batched": serving.latency_summary(srv.run(burst, realtime=False)),
                        "plain": serving.latency_summary(plain.run(burst, realtime=False))}
    out["server_reserved_gb"] = srv.reserved_bytes() / 1e9
    srv.close()
    plain.close()
    return out


def differentiation_report(dev):
    """Differentiable path on 200,000 Gaussians at 1024x768 (loss = L1 + 0.2 (1 - SSIM)
    through torch.autograd): forward and backward times (CUDA events, median of 5 after
    2 warm-ups) and device memory with recomputed vs stored transmittance."""
    import torch
    from msplat_street_b200 import autograd as ag
    from msplat_street_b200 import scenes
    from msplat_street_b200.backend import GaussianParams
    from msplat_street_b200.workloads import BACKGROUND

    g = scenes.random_gaussians(200_000, 21)
    cam = scenes.small_camera(1024, 768, 1000.0, 3.0)
    with torch.no_grad():
        gt = ag.render(GaussianParams.from_numpy(scenes.random_gaussians(200_000, 22), dev), cam, BACKGROUND)
    out = {"case": "200k Gaussians, 1024x768, L1+0.2(1-SSIM)"}
    for mode, cap in (("recompute", 0), ("store", 256)):
        ag.set_transmittance_mode(mode, cap or 256)
        ag._POOL.clear()
        torch.cuda.empty_cache()
        torch.cuda.reset_peak_memory_stats(dev)
        fw, bw = [], []
        for it in range(7):
            p = GaussianParams(*[torch.from_numpy(a).to(dev).requires_grad_(True) for a in g.arrays()])
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            loss = ag.ssim_l1_loss(ag.render(p, cam, BACKGROUND), gt)
            e1.record()
            loss.backward()
            e2.record()
            torch.cuda.synchronize()
            if it >= 2:
                fw.append(e0.elapsed_time(e1))
                bw.append(e1.elapsed_time(e2))
        out[mode] = {"forward_ms": statistics.median(fw), "backward_ms": statistics.median(bw),
                     "frame_bytes": ag.pool_device_bytes(),
                     "torch_peak_bytes": int(torch.cuda.max_memory_allocated(dev)),
                     "peak_hbm_bytes": ag.pool_device_bytes() + int(torch.cuda.max_memory_allocated(dev))}
    ag.set_transmittance_mode("recompute")
    ag._POOL.clear()
    return out


def chunked_report(dev):
    """One-pass vs depth-chunked compositing (512-long pieces, the Metal backend's
    small-frame path) on frames of 256 tiles: mean ms per call over 10 calls after 3
    warm-ups (CUDA events). Renders of a 1 M-Gaussian scene drawn from the serving
    distributions, opaque as drawn and with every opacity logit at -4.5 (alpha <= 0.011:
    no pixel saturates, so one pass walks whole lists), and a 300 k-Gaussian training
    step."""
    import torch
    from msplat_street_b200 import scenes, serving
    from msplat_street_b200.backend import AdamState, Context, GaussianParams
    from msplat_street_b200.workloads import BACKGROUND

    def mean_ms(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    cam = scenes.small_camera(256, 256, 230.0, 3.0)
    out = {"frame": "256x256 (256 tiles)", "chunk_len": 512}
    p = serving.random_scene_tensors(1_000_000, 7, device=dev)
    faint = GaussianParams(p.means, p.scales, p.quats, p.features_dc, p.features_rest,
                           torch.full_like(p.opacities, -4.5))
    for name, scene in (("render_1m", p), ("render_1m_faint", faint)):
        row = {}
        for mode in ("off", "on"):
            ctx = Context(chunked=mode)
            row["one_pass_ms" if mode == "off" else "chunked_ms"] = mean_ms(lambda: ctx.render(scene, cam, BACKGROUND))
            row["intersections"] = ctx.num_isects()
        out[name] = row
    g = scenes.random_gaussians(300_000, 11, log_scale_mean=-3.0)
    gt = torch.rand((256, 256, 3), device=dev)
    row = {}
    for mode in ("off", "on"):
        ctx = Context(chunked=mode)
        q = GaussianParams.from_numpy(g, dev)
        adam = AdamState.zeros_like(q, [1.6e-4, 5e-3, 1e-3, 2.5e-3, 2.5e-3, 0.05])
        stats = tuple(torch.zeros(g.n, device=dev) for _ in range(3))
        row["one_pass_ms" if mode == "off" else "chunked_ms"] = mean_ms(
            lambda: ctx.train_step(q, adam, cam, BACKGROUND, gt, stats))
    out["train_step_300k"] = row
    return out


class TargetPrefetch:
    """Each step's target copied from pinned host memory on a copy stream, one step
    ahead, so the upload of step i + 1 overlaps step i's kernels (a production input
    pipeline). The camera schedule is the trainer's own: permutations are drawn from
    its generator in the same sequence, only earlier."""

    def __init__(self, trainer, host_targets, dev):
        import torch
        self.tr, self.host, self.dev = trainer, host_targets, dev
        self.stream = torch.cuda.Stream(device=dev)
        self.pending = self._issue(1)

    def _camera(self, ahead: int) -> int:
        tr = self.tr
        while len(tr._order) < ahead:  # the permutation the trainer would draw next
            tr._order = list(tr._rng.permutation(len(tr.ds.views))) + tr._order
        return tr._order[-ahead]

    def _issue(self, ahead: int):
        import torch
        ci = self._camera(ahead)
        with torch.cuda.stream(self.stream):
            t = self.host[ci].to(self.dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        return t, ev

    def next(self):
        """The next step's target, ready on the current stream; starts the following
        step's upload."""
        import torch
        t, ev = self.pending
        cur = torch.cuda.current_stream(self.dev)
        cur.wait_event(ev)
        t.record_stream(cur)
        self.pending = self._issue(2)
        return t


def launches_per_step(n_isect: float, n_gauss: float = 1e5) -> float:
    """Kernels one plain training step launches: project, depth keys, the depth sort
    (4 passes of hist + scatter, plus a 3-kernel scan per pass above 131,072
    Gaussians), tile counts gathered, their 3-kernel scan, offsets scattered, emission,
    the tile sort (2 passes of hist + 3-kernel scan + scatter for 2048 tiles), ranges,
    map, raster forward, SSIM, loss finalize, raster backward, backward/Adam."""
    tiles_bits = 11  # 1024x512 -> 2048 tiles
    tile_passes = (tiles_bits + 7) // 8
    depth_sort = 4 * (2 if n_gauss <= 131072 else 5)
    return 1 + 1 + depth_sort + 1 + 3 + 1 + 1 + tile_passes * 5 + 1 + 1 + 1 + 1 + 1 + 1 + 1


# DRAM bytes read + written by one launch of the rasterizer backward, from an ncu
# capture of the street step's first timed launch (1.86 M intersections), and the
# intersections it processed; the run scales it by its own intersections.
NCU_RAST_BWD = {"dram_bytes": 16.66e6 + 0.87e6, "isects": 1.86e6}

SM_COUNT, FP32_LANES = 148, 128
NPIX = 1024 * 512
# FP32 operations per evaluated (pixel, Gaussian) pair: forward sigma, alpha and the
# colour / transmittance update; backward recovery, v_alpha, the sigma, conic, xy,
# colour and opacity gradients
FWD_OPS_PER_PAIR, BWD_OPS_PER_PAIR = 20.0, 50.0


def stage_bytes(n_isects: float, n_gauss: float) -> dict:
    """Algorithmic bytes per step of each stage (each input read once, each output
    written once):
     proj_sh_fwd: 236 B of parameters read + 48 B splat record, radius, box, tile
       count (76 B) written per Gaussian;
     bin_sort: key emission 12 B per intersection, the tile sort's passes 24 B per
       intersection per pass (2 passes for 2048 tiles), ranges and map 8 + 8 B;
     rast_fwd: splat record 48 B + id 4 B per intersection, 20 B per pixel written;
     loss_fwd_bwd: 36 B per pixel (render + target read, gradient written);
     rast_bwd: 48 + 4 B per intersection read + 36 B slot written, 32 B per pixel read;
     proj_sh_bwd_adam: per Gaussian 11 dense parameters x 3 arrays read + written
       (264 B) + SH 48 x 3 x 2 (1152 B), 36 B slot per intersection read."""
    return {
        "proj_sh_fwd": n_gauss * (236 + 76),
        "bin_sort": n_isects * (12 + 2 * 24 + 16),
        "rast_fwd": n_isects * 52 + NPIX * 20,
        "loss_fwd_bwd": NPIX * 36,
        "rast_bwd": n_isects * 88 + NPIX * 32,
        "proj_sh_bwd_adam": n_gauss * (264 + 1152) + n_isects * 36,
    }


def fp32_peak_gflops(sm_mhz) -> float:
    """148 SMs x 128 FP32 lanes x 2 (a fused multiply-add) x the sampled SM clock."""
    mhz = float(sm_mhz) if sm_mhz else 1965.0
    return SM_COUNT * FP32_LANES * 2 * mhz * 1e6 / 1e9


def roofline(stages, n_isects, n_gauss, peaks, peak_kind, pairs=None, sm_mhz=None):
    """The dominant stage by time against the measured HBM copy bandwidth, with its
    algorithmic bytes (stage_bytes) over its live CUDA-event duration. For the
    rasterizers, which are bound by instruction issue rather than HBM, `compute` adds
    the FP32 fraction: the reference loops' (pixel, Gaussian) pairs (counted on the
    device each step) x the operations per pair over the FP32 peak at the sampled
    clock."""
    if not stages:
        return None
    per = {k: v[0] / max(v[1], 1) for k, v in stages.items()}
    dom = max(per, key=per.get)
    isect = float(np.mean(n_isects)) if n_isects else 0.0
    algo = stage_bytes(isect, n_gauss).get(dom, 0.0)
    ms = per[dom]
    achieved = algo / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
    out = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
           "avg_ms": ms, "algorithmic_bytes": algo}
    if dom == "rast_bwd":
        # the splat records' re-reads hit L2, so DRAM traffic is well below the
        # algorithmic bytes
        out["traffic"] = NCU_RAST_BWD["dram_bytes"] * isect / NCU_RAST_BWD["isects"]
        out["traffic_source"] = "ncu capture of one launch (street step, 1.86 M intersections), scaled by intersections"
    if dom in ("rast_fwd", "rast_bwd") and pairs:
        k = 0 if dom == "rast_fwd" else 1
        ops = FWD_OPS_PER_PAIR if dom == "rast_fwd" else BWD_OPS_PER_PAIR
        gflops = float(np.mean([p[k] for p in pairs])) * ops / (ms * 1e-3) / 1e9
        pk = fp32_peak_gflops(sm_mhz)
        out["compute"] = {"bound": "fp32 issue", "achieved": gflops, "peak": pk, "unit": "GFLOP/s",
                          "frac": gflops / pk, "ops_per_pair": ops,
                          "peak_source": "computed: 148 SMs x 128 lanes x 2 x sampled SM clock"}
    return out


def throughput(stages, n_isects, n_gauss, pairs, peaks, peak_kind, sm_mhz) -> dict:
    """Per-stage rates of the timed window in the units of the path: Gaussians/s
    projected, Mpix/s composited, (pixel, Gaussian) pairs/s and the FP32 fraction of the
    rasterizers, and every stage's algorithmic HBM GB/s against the measured peak."""
    per = {k: v[0] / max(v[1], 1) for k, v in stages.items()}
    isect = float(np.mean(n_isects)) if n_isects else 0.0
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
    fwd_pairs = float(np.mean([p[0] for p in pairs])) if pairs else 0.0
    bwd_pairs = float(np.mean([p[1] for p in pairs])) if pairs else 0.0
    pk = fp32_peak_gflops(sm_mhz)
    out = {"gaussians": n_gauss, "isects": isect, "pairs_fwd": fwd_pairs, "pairs_bwd": bwd_pairs,
           "fp32_peak_gflops": pk, "hbm_peak_gbs": peak, "peak_source": peak_kind}
    if per.get("proj_sh_fwd"):
        out["gaussians_per_s_projected"] = n_gauss / (per["proj_sh_fwd"] * 1e-3)
    if per.get("rast_fwd"):
        t = per["rast_fwd"] * 1e-3
        out["mpix_per_s_composited"] = NPIX / t / 1e6
        out["pairs_per_s_fwd"] = fwd_pairs / t
        out["fp32_frac_fwd"] = fwd_pairs * FWD_OPS_PER_PAIR / t / 1e9 / pk
    if per.get("rast_bwd"):
        t = per["rast_bwd"] * 1e-3
        out["pairs_per_s_bwd"] = bwd_pairs / t
        out["fp32_frac_bwd"] = bwd_pairs * BWD_OPS_PER_PAIR / t / 1e9 / pk
    hbm = {}
    for k, b in stage_bytes(isect, n_gauss).items():
        if per.get(k):
            gbs = b / (per[k] * 1e-3) / 1e9
            hbm[k] = {"ms": per[k], "bytes": b, "gbs": gbs, "frac": gbs / peak}
    out["hbm"] = hbm
    return out


SCHEDULE_WINDOWS = ((500, 519), (1000, 1019), (1500, 1519), (1980, 1999))


def schedule_sample(trainer, ctx, flush, dev, windows=SCHEDULE_WINDOWS) -> list:
    """Continues the timed trainer through the schedule and times 20-step windows at
    its landmarks -- the first densification (step 500), the last (1000, where
    refinement stops and SH degree 1 begins), mid-run and the end -- each step
    device-timed with CUDA events like the headline window, L2 flushed between
    steps."""
    import torch
    out = []
    for a, b in windows:
        if trainer.iteration >= a or b > trainer.cfg.iterations:
            continue
        while trainer.iteration < a - 1:
            trainer.step()
        torch.cuda.synchronize()
        n0, dens, ms, isects = trainer.splat_count, [], [], []
        for _ in range(b - a + 1):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            before = trainer.splat_count
            e0.record()
            st = trainer.step()
            e1.record()
            isects.append(ctx.num_isects())
            if st.splat_count != before:
                dens.append(st.iteration)
            ms.append((e0, e1))
        torch.cuda.synchronize()
        per = [x.elapsed_time(y) for x, y in ms]
        t = sum(per)
        slow = int(np.argmax(per))
        out.append({"iterations": [a, b], "ms_per_step": t / len(ms), "iters_per_s": len(ms) / (t / 1e3),
                    "gaussians": [n0, trainer.splat_count], "sh_degree": trainer.degrees_to_use(),
                    "densify_steps": dens, "isects_mean": float(np.mean(isects)),
                    "slowest_step": {"iteration": a + slow, "ms": per[slow]}})
    return out


def knn_rate(trainer, ctx, reps: int = 5) -> dict:
    """Exact 3-NN mean distance (the scale init) over the workload's initial point
    cloud: points/s and point-distance evaluations/s (counted on the device), CUDA
    events around each call."""
    import torch
    pts = torch.from_numpy(trainer.ds.points).cuda()
    ctx.knn3_mean_dist(pts)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.knn3_mean_dist(pts)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = statistics.median(ts)
    evals = int(ctx.frame("knn_evals").view(torch.int64)[0])  # the last call's (every call's) count
    return {"points": int(pts.shape[0]), "ms": ms, "points_per_s": pts.shape[0] / (ms * 1e-3),
            "distance_evals": evals, "distance_evals_per_s": evals / (ms * 1e-3)}


PROFILE_CASES = ("sort", "ssim", "adam", "densify", "render")


def profile_case(name: str, dev, runs: int = 2, shape=None) -> dict:
    """One stage at a size larger than the 126 MB L2, run `runs` times (default twice:
    the second launch is the one an ncu capture takes with -s 1 -c 1 on the stage's
    kernel), for the DRAM traffic and achieved bandwidth of that kernel; "stage_ms" holds
    the context's CUDA-event stage times per run over the runs after the first:
      sort     stable radix sort of 32 M (u64 key, i32 value) pairs, 40 key bits (5 passes)
      ssim     fused L1 + SSIM forward and backward of a 4096 x 4096 render
      adam     backward/Adam of a training step over 1 M Gaussians (SH degree 3)
      densify  clone / split / prune + compaction of 500 k Gaussians (capacity 2 M)
      render   a batched render (the serving path) of a 3 M-Gaussian scene drawn from
               the serving distributions at 1920 x 1080 from 5 m"""
    import torch
    from msplat_street_b200 import autograd, scenes
    from msplat_street_b200.backend import AdamState, Context, GaussianParams

    ctx = Context()
    if shape is not None:
        ctx.set_raster_shape(shape)
    g = torch.Generator(device=dev).manual_seed(7)
    out = {"case": name}
    runs = max(2, runs)

    walls = []

    def timed(it):  # stage timing from the second run on; wall time of each run
        torch.cuda.synchronize()
        if walls and walls[-1] < 0:
            walls[-1] += time.perf_counter()
        if it == 1:
            ctx.enable_stage_timing(True)
            ctx.drain_stage_times()
        walls.append(-time.perf_counter())
        return it

    if name == "sort":
        n = 32 << 20
        src = torch.randint(0, 1 << 40, (n,), device=dev, dtype=torch.int64, generator=g)
        for it in range(runs):
            keys = src.clone()
            vals = torch.arange(n, device=dev, dtype=torch.int32)
            timed(it)
            ctx.radix_sort(keys, vals, 40)
        out.update(pairs=n, key_bits=40, bytes_per_pair_pass=24)
    elif name == "ssim":
        h = w = 4096
        img = torch.rand((h, w, 3), device=dev, generator=g)
        gt = torch.rand((h, w, 3), device=dev, generator=g)
        for it in range(runs):
            timed(it)
            loss = autograd.ssim_l1_loss(img.requires_grad_(), gt)
            loss.backward()
            img.grad = None
        out.update(pixels=h * w, bytes_per_pixel=36)
    elif name == "adam":
        n = 1 << 20
        p = GaussianParams.from_numpy(scenes.random_gaussians(n, 3, log_scale_mean=-5.0), dev)
        cam = scenes.small_camera(512, 512, 600.0)
        gt_img = torch.rand((512, 512, 3), device=dev, generator=g)
        adam = AdamState.zeros_like(p, [1.6e-4, 5e-3, 1e-3, 2.5e-3, 1.25e-4, 0.05])
        stats = tuple(torch.zeros(n, device=dev) for _ in range(3))
        for it in range(runs):
            timed(it)
            ctx.train_step(p, adam, cam, np.zeros(3, np.float32), gt_img, stats)
        torch.cuda.synchronize()
        vis = int((ctx.frame("radii") > 0).sum())
        out.update(gaussians=n, visible=vis, isects=ctx.num_isects(), dense_bytes_per_gaussian=264,
                   sh_bytes_per_visible=1152, slot_bytes_per_isect=40)
    elif name == "densify":
        n, cap = 500_000, 2_000_000  # room for every Gaussian to be split and cloned
        src = scenes.random_gaussians(n, 4, log_scale_mean=-4.0, log_scale_std=1.5)
        strides = [3, 3, 4, 3, 45, 1]
        for it in range(runs):
            bufs = []
            for a, st in zip(src.arrays(), strides):
                b = torch.zeros((cap, st), device=dev)
                b[:n] = torch.from_numpy(a.reshape(n, st)).to(dev)
                bufs.append(b)
            m1 = [torch.rand((cap, st), device=dev, generator=g) for st in strides]
            m2 = [torch.rand((cap, st), device=dev, generator=g) for st in strides]
            gn = torch.rand(n, device=dev, generator=g) * 4e-3
            vc = torch.randint(1, 4, (n,), device=dev, generator=g).float()
            ms = torch.rand(n, device=dev, generator=g) * 0.3
            timed(it)
            new_n = ctx.densify(n, bufs, m1, m2, gn, vc, ms, 512.0, 1234)
        out.update(gaussians=n, capacity=cap, new_gaussians=new_n, floats_per_gaussian=59, arrays=3)
    elif name == "render":
        from msplat_street_b200 import serving
        from msplat_street_b200.backend import BatchItem
        from msplat_street_b200.workloads import BACKGROUND
        p = serving.random_scene_tensors(3_000_000, 7, device=dev)
        cam = scenes.sphere_camera(np.random.default_rng(3), 1920, 1080, radius=5.0)
        for it in range(runs):
            timed(it)
            ctx.render_batch([BatchItem(p, cam, BACKGROUND)])
        torch.cuda.synchronize()
        out.update(gaussians=3_000_000, resolution="1920x1080", isects=ctx.num_isects())
    torch.cuda.synchronize()
    if walls and walls[-1] < 0:
        walls[-1] += time.perf_counter()
    out["run_wall_ms"] = [round(1e3 * w, 3) for w in walls]
    st = ctx.drain_stage_times()
    ctx.enable_stage_timing(False)
    out["stage_ms"] = {k: round(v[0] / max(1, runs - 1), 4) for k, v in st.items() if v[1] > 0}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1990)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quick", action="store_true", help="device-timed pass only (no e2e, no CPU baseline)")
    ap.add_argument("--serving-seconds", type=float, default=1.0,
                    help="length of each Poisson request stream in the serving report (0 = skip)")
    ap.add_argument("--no-batching", action="store_true", help="skip the batched-training report")
    ap.add_argument("--profile-case", choices=PROFILE_CASES,
                    help="run one stage at a size larger than L2 (for an ncu capture) and exit")
    ap.add_argument("--case-runs", type=int, default=2, help="runs of the --profile-case stage (at least 2)")
    ap.add_argument("--raster-shape", type=int, default=None,
                    help="forward rasterizer block shape (0: 16x16, 1: 16x8, 2: 8x8; default: the library's)")
    args = ap.parse_args(argv)
    if args.profile_case:
        import torch
        print(json.dumps(profile_case(args.profile_case, torch.device("cuda", 0), args.case_runs, args.raster_shape)))
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
