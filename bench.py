#!/usr/bin/env python
"""Benchmark: train iter/s (fwd + bwd + Adam) of the 1M-Gaussian, 8-views-per-step
workload (batched multi-view step vs the plain per-view path), on B200.

Workload (synthetic, seeded; no dataset is involved): 1M Gaussians with means
U[-2, 2]^3, log-scales N(-4, 0.5), normalised N(0, 1) quaternions, opacity
logits N(0, 1), SH degree 3 (DC N(0, 0.3), rest N(0, 0.05)); 128 cameras on a
radius-5 Fibonacci sphere cycling through 1600x1064, 1280x720 and 960x540
(fx = fy = 1.25 * width); 8 views per step picked with the reference's
xorshift64 camera shuffle (src/pipeline/mod.rs:224-230); targets rendered from
the scene with means perturbed by N(0, 0.02).

`python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]`
prints one JSON line (rank 0). Under torchrun (N > 1) every rank trains its own
8 views per step and the gradients are summed with an NCCL all-reduce before a
replicated Adam step (view-parallel data parallelism, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "train iter/s (fwd+bwd+Adam) batched vs plain GPU path, 1M Gaussians, at tol"
UNIT = "iter/s"
WORKLOAD = "1M Gaussians, SH3, 8 views/step from 128 sphere cameras {1600x1064, 1280x720, 960x540}"


def xorshift_views(state: list, n_cams: int, k: int) -> list[int]:
    """src/pipeline/mod.rs:224-230: x ^= x << 13; x ^= x >> 7; x ^= x << 17; x % n."""
    out = []
    m = (1 << 64) - 1
    for _ in range(k):
        x = state[0]
        x ^= (x << 13) & m
        x ^= x >> 7
        x ^= (x << 17) & m
        state[0] = x
        out.append(x % n_cams)
    return out


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--scale", type=float, default=1.0, help="fraction of the 1M Gaussians (smaller cases for profiling)")
    p.add_argument("--views", type=int, default=8)
    p.add_argument("--plain-steps", type=int, default=None)
    p.add_argument("--cpu-budget", type=float, default=45.0,
                   help="seconds of timed CPU work for the reference arm (whole iterations; at least one)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--tile", default="16x16")
    p.add_argument("--batch", type=int, default=128)
    p.add_argument("--ppt", type=int, default=2, help="pixels per thread of the forward blend (1 or 2; the backward takes twice as many)")
    p.add_argument("--no-autotune", action="store_true", help="keep --tile/--batch/--ppt instead of autotuning")
    p.add_argument("--no-variants", action="store_true", help="skip the recompute vs store-all backward measurement")
    p.add_argument("--no-rows", action="store_true", help="skip the preview / target / model-file row measurements")
    p.add_argument("--rows-only", action="store_true", help="measure only those rows (at --scale) and exit")
    return p.parse_args()


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        # NVML read every 10 ms from a thread (the timed region can be a few
        # hundred ms); nvidia-smi at its 200 ms floor otherwise. Read-only.
        self.samples, self.nvml = [], None
        try:
            import threading

            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.stop_ev = threading.Event()

            def run():
                while not self.stop_ev.is_set():
                    try:
                        mhz = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((mhz, [k for k, b in bits.items() if r & b]))
                    except Exception:
                        pass
                    self.stop_ev.wait(0.01)

            self.nvml = threading.Thread(target=run, daemon=True)
            self.nvml.start()
            return
        except Exception:
            self.nvml = None
        try:
            import tempfile

            fd, self.path = tempfile.mkstemp(prefix=f"rgs_clocks_gpu{self.device}_", suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                                          "-i", str(self.device)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.nvml is not None:
            self.stop_ev.set()
            self.nvml.join(timeout=2)
            sm = [m for m, _ in self.samples]
            reasons = sorted({r for _, rs in self.samples for r in rs})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def build_workload(scale: float):
    from rgsplat_b200 import scenes

    cfg = scenes.config(3, n=max(1000, int(round(1_000_000 * scale))))
    g = scenes.make_gaussians(cfg)
    return cfg, g


def render_targets(R, scenes, cfg, g, ctx):
    """RGBA targets of every camera, rendered on the GPU from the perturbed scene."""
    tr = R.Trainer(scenes.perturbed(g, cfg.seed + 1), cfg.cameras, ctx=ctx)
    targets = []
    for i, c in enumerate(cfg.cameras):
        rgb = tr.render(i)
        t = np.empty((c.height, c.width, 4), np.float32)
        t[..., :3] = rgb
        t[..., 3] = 1.0
        targets.append(t)
    return targets


def algorithmic_bytes(stage: str, n: int, views: int, pairs: int, pixels: int, visible: int, entries: int) -> float:
    """Per-step algorithmic HBM bytes of a stage: what an ideal kernel must
    move, each datum once (S = views * n slots; `visible` = slots with at
    least one tile pair; `entries` = (supertile, slot) entries; a splat record
    is 48 B, a Gaussian 240 B)."""
    S = views * n
    if stage == "project":
        return n * 240.0 + S * (48 + 4 + 8 + 8 + 4 + 4)           # params once; record, count, rect, spans, key, id per slot
    if stage == "depth_sort":
        # compaction: count + key per slot read; key, slot, supertile count + rect per visible slot
        # written; sort: (key, slot) read + written once
        return S * 8.0 + visible * (8 + 12) + visible * 8.0 * 2
    if stage == "emit":
        # two count scans (order + count), then order + supertile rect per visible slot; entries written
        return visible * (8 + 8) + visible * (4 + 8) + entries * 8.0
    if stage == "supertile_sort":
        return entries * 8.0 * 2                                   # (supertile, slot) read + written once
    if stage == "tile_lists":
        # entries read; rect + packed spans per visible slot; one slot per pair written
        return entries * 8.0 + visible * (8 + 8) + pairs * 4.0
    if stage == "forward":
        return pairs * 4.0 + visible * 48.0 + pixels * 20.0        # pair list, records once; rgb, T, last written
    if stage == "loss":
        return pixels * (12.0 + 16.0 + 12.0)                       # rendered, target read; dL/dpixel written
    if stage == "backward":
        return pixels * 20.0 + pairs * 4.0 + visible * (48.0 + 48.0)  # caches, pair list, records; accumulators
    if stage == "geometry_adam":
        return n * (240.0 * 3 * 2 + 8) + S * 4.0 + visible * (48.0 + 48.0)  # params, m1, m2 r+w; counts; acc + record
    return 0.0


def profiled_traffic(kernel_file: str):
    """DRAM bytes per launch of a kernel from its committed ncu summary."""
    try:
        txt = open(os.path.join(ROOT, "profiles", kernel_file)).read()
        m = re.search(r"dram_bytes_per_launch:\s*(\d+)", txt)
        return int(m.group(1)) if m else None
    except OSError:
        return None


def profiled_issue_active(kernel: str):
    """Fraction of issue slots the packed blend kernel kept busy, from the
    committed ncu pipe-mix table (quarter-size capture of the same launch
    shape; columns: forward scalar, forward packed, backward scalar, backward
    packed)."""
    col = {"k_blend_fwd": 3, "k_blend_bwd": 5}.get(kernel)
    try:
        for line in open(os.path.join(ROOT, "profiles", "blend_pipes_250k_8views.md")):
            if col and line.startswith("| issue slots active |"):
                return round(float(line.split("|")[col].strip().rstrip("%").strip()) / 100.0, 3)
    except (OSError, ValueError, IndexError):
        pass
    return None


def measure_backward_variants(R, scenes, device: int, reps: int = 5) -> dict:
    """Differentiation workload (50k Gaussians, one 512x512 view): the
    recompute-from-final-T backward against the store-all-T variant, blend
    kernel times (median of reps, CUDA events), the blend state each keeps, and
    the device memory each needs: the high-water mark of a fresh context's
    buffers over its first call (everything the call allocated, parameters and
    pair buffers included)."""
    cfg = scenes.config(2)
    g = scenes.make_gaussians(cfg)
    cam = cfg.cameras[0]
    rgb = R.render_color(scenes.perturbed(g, cfg.seed + 1), cam, ctx=R.Context(device=device))
    target = np.concatenate([rgb, np.ones((cam.height, cam.width, 1), np.float32)], axis=2)
    out = {"workload": "50k Gaussians, one 512x512 view"}
    for name, store in (("recompute", False), ("store_all", True)):
        ctx = R.Context(device=device)
        first = R.render_and_backward_variant(g, cam, target, store_all=store, ctx=ctx)[2]
        mem = ctx.memory()
        reps_out = [R.render_and_backward_variant(g, cam, target, store_all=store, ctx=ctx)[2] for _ in range(reps)]
        out[name] = {"forward_ms": round(float(np.median([r["forward_ms"] for r in reps_out])), 4),
                     "backward_ms": round(float(np.median([r["backward_ms"] for r in reps_out])), 4),
                     "blend_state_bytes": int(first["state_bytes"]), "pairs": int(first["pairs"]),
                     "peak_device_bytes": mem["peak_bytes"]}
        ctx.close()
    return out


def measure_next_rows(R, g, cam, device: int, reps: int = 5, cpu: bool = True) -> dict:
    """The rows either side of the training step, each through its public call
    with host buffers (host<->device copies and, for the model files, the file
    write / read inside the time): median of reps after one untimed call, and
    the oracle on the host cores for the same input (one call each)."""
    import tempfile

    ctx = R.Context(device=device)
    rng = np.random.default_rng(9)
    img = rng.integers(0, 256, size=(cam.height, cam.width, 4), dtype=np.uint8)
    px = cam.width * cam.height
    pts = rng.normal(size=(g.shape[0], 3)) * np.array([4.0, 2.0, 3.0])
    cols = rng.integers(0, 256, size=(g.shape[0], 3), dtype=np.uint8)
    tmp = tempfile.mkdtemp(prefix="rgs_rows_")
    ply, splat = os.path.join(tmp, "m.ply"), os.path.join(tmp, "m.splat")
    n = g.shape[0]
    preview = R.Trainer(g, [cam])
    rows = {
        "rasterize_srgb8": (lambda: R.rasterize(g, cam, srgb8=True, ctx=ctx), px * 4,
                            f"cpu::rasterize + to_u8_srgb, {n} Gaussians, one {cam.width}x{cam.height} view"),
        "trainer_rasterize_srgb8": (lambda: preview.rasterize(0, srgb8=True), px * 4,
                                    f"the same preview of a trainer's device-resident Gaussians (no upload)"),
        "target_srgb8_to_linear": (lambda: R.srgb8_to_linear(img, ctx=ctx), px * 20,
                                   f"load_target conversion, {cam.width}x{cam.height} RGBA8 -> linear f32"),
        "save_ply": (lambda: R.save_ply(g, ply, ctx=ctx), n * 248, f"io::ply::save_ply, {n} Gaussians"),
        "save_splat": (lambda: R.save_splat(g, splat, ctx=ctx), n * 32, f"io::ply::save_splat, {n} Gaussians"),
        "load_ply": (lambda: R.load_ply(ply, ctx=ctx), n * 248, f"io::ply::load_ply, {n} Gaussians"),
        "gaussians_from_sfm": (lambda: R.gaussians_from_sfm(pts, cols, ctx=ctx), n * (27 + 236),
                               f"gaussians_from_sfm + KNN scales, {n} SfM points"),
    }
    out = {}
    for name, (fn, nbytes, what) in rows.items():
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        ms = float(np.median(ts)) * 1e3
        out[name] = {"workload": what, "ms": round(ms, 3), "user_bytes": int(nbytes),
                     "user_gbs": round(nbytes / (ms / 1e3) / 1e9, 2)}
    if cpu:
        import oracle as O

        threads = O.set_threads(os.cpu_count() or 1)
        ply_bytes = open(ply, "rb").read()
        oracle_rows = {
            "rasterize_srgb8": lambda: O.to_u8_srgb(O.rasterize(g, cam)),
            "trainer_rasterize_srgb8": lambda: O.to_u8_srgb(O.rasterize(g, cam)),
            "target_srgb8_to_linear": lambda: O.srgb8_to_linear(img.reshape(-1, 4)),
            "save_ply": lambda: open(ply + ".o", "wb").write(O.save_ply_bytes(g)),
            "save_splat": lambda: open(splat + ".o", "wb").write(O.save_splat_bytes(g)),
            "load_ply": lambda: O.load_ply_bytes(open(ply, "rb").read()),
            "gaussians_from_sfm": lambda: O.gaussians_from_sfm(pts, cols),
        }
        for name, fn in oracle_rows.items():
            t0 = time.perf_counter()
            fn()
            out[name]["oracle_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
            out[name]["oracle_threads"] = threads if name.endswith("rasterize_srgb8") else 1
        del ply_bytes
    for f in (ply, splat, ply + ".o", splat + ".o"):
        if os.path.exists(f):
            os.remove(f)
    os.rmdir(tmp)
    return out


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# the workload both arms run: static description and view schedule
# ---------------------------------------------------------------------------
def workload_config(cfg, n: int, views: int, world: int) -> dict:
    """What the timed step is: identical in both arms' lines (nothing measured)."""
    sizes = sorted({(c.width, c.height) for c in cfg.cameras}, reverse=True)
    return {"workload": WORKLOAD, "n_gaussians": int(n), "views_per_step": int(views), "cameras": len(cfg.cameras),
            "resolutions": [f"{w}x{h}" for w, h in sizes], "sh_degree": 3, "precision": "f32",
            "view_schedule": "xorshift64 from 0x9E3779B97F4A7C15 (rank-offset seed per rank), warm-up view sets "
                             "first, then the timed ones",
            "parallelism": f"view-dp{world}",
            "l2": "inputs larger than L2 (240 MB params + 480 MB moments + targets)"}


def view_schedule(n_cams: int, views: int, warmup: int, steps: int, rank: int):
    """(all view sets, the timed ones) of one rank: warm-up sets, then `steps` sets."""
    from rgsplat_b200 import dp

    st = [dp.rank_seed(0x9E3779B97F4A7C15, rank)]
    schedule = [xorshift_views(st, n_cams, views) for _ in range(warmup + max(steps, 1))]
    return schedule, schedule[warmup:]


# ---------------------------------------------------------------------------
# reference arm: the oracle (C++ restatement of the reference CPU path) on host cores
# ---------------------------------------------------------------------------
def oracle_iterations(g, cfg, view_sets, target_fn, budget_s: float, max_iters: int, warmup_views: int = 0):
    """Whole training iterations of the reference path on the host cores: per
    view set, render_and_backward of every view (gradients summed over the
    views), then one Adam step with grad_denom += views, parameters updated in
    place between iterations. Targets are made before each iteration's clock
    starts. Runs at least one iteration and stops at max_iters or once
    budget_s has been spent. Returns (seconds per iteration, iterations,
    threads, warm-up calls)."""
    import oracle as O

    threads = O.set_threads(os.cpu_count() or 1)
    gg = np.ascontiguousarray(g).copy()
    state = O.AdamState(gg.shape[0])
    tcfg = O.TrainConfig()
    for k in range(warmup_views):  # untimed single-view calls: threads and caches warm
        v = view_sets[0][k % len(view_sets[0])]
        O.render_and_backward(gg, cfg.cameras[v], target_fn(v), (0.0, 0.0, 0.0), 0.2)
    times = []
    spent = 0.0
    for vs in view_sets[: max(max_iters, 1)]:
        tg = {v: target_fn(v) for v in vs}
        t0 = time.perf_counter()
        total = None
        for v in vs:
            out = O.render_and_backward(gg, cfg.cameras[v], tg[v], (0.0, 0.0, 0.0), 0.2)
            total = out.grads if total is None else total + out.grads
        O.adam_step(gg, total, state, tcfg)
        state.grad_denom += np.uint32(len(vs) - 1)
        times.append(time.perf_counter() - t0)
        spent += times[-1]
        if spent >= budget_s:
            break
    return float(np.mean(times)), len(times), threads, warmup_views


def oracle_targets(cfg, g):
    """Targets rendered by the oracle from the perturbed scene (bit-identical to
    the GPU arm's, which renders them with the library), cached per camera."""
    import oracle as O
    from rgsplat_b200 import scenes

    tg = scenes.perturbed(g, cfg.seed + 1)
    cache = {}

    def target(v):
        if v not in cache:
            rgb, _, _ = O.render_color(tg, cfg.cameras[v])
            cache[v] = np.concatenate([rgb, np.ones((cfg.cameras[v].height, cfg.cameras[v].width, 1), np.float32)], axis=2)
        return cache[v]

    return target


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    cfg, g = build_workload(args.scale)
    _, timed_views = view_schedule(len(cfg.cameras), args.views, args.warmup, args.steps, 0)
    s_iter, iters, threads, warm = oracle_iterations(g, cfg, timed_views, oracle_targets(cfg, g), args.cpu_budget, args.steps,
                                                     warmup_views=min(max(args.warmup, 0), 3))
    value = 1.0 / s_iter
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": iters,
        "steps_requested": args.steps, "warmup": warm, "views_sampled": iters * args.views,
        "ms_per_step": s_iter * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": workload_config(cfg, g.shape[0], args.views, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{iters} whole iterations ({args.views} x render_and_backward + one Adam step, "
                                   f"{s_iter:.2f} s each) on the first {iters} of the GPU arm's timed view sets, "
                                   f"after {warm} untimed single-view calls; the --steps request is cut at "
                                   f"{args.cpu_budget:.0f} s of timed CPU work"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    import rgsplat_b200 as R
    from rgsplat_b200 import scenes

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local_rank))

    if args.rows_only:
        # only the rows either side of the step (preview, target upload, model
        # files, SfM initialisation), at this --scale: a small case to profile
        if rank == 0:
            cfg, g = build_workload(args.scale)
            rows = measure_next_rows(R, g, cfg.cameras[0], local_rank, reps=1, cpu=not args.no_cpu_baseline)
            print(json.dumps({"next_rows": rows, "n_gaussians": int(g.shape[0])}), flush=True)
        return
    tw, th = (int(x) for x in args.tile.split("x"))
    ctx = R.Context(device=local_rank, tile=(tw, th), batch=args.batch, pixels_per_thread=args.ppt)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    cfg, g = build_workload(args.scale)
    n = g.shape[0]
    V = args.views
    with torch.cuda.stream(stream):
        targets = render_targets(R, scenes, cfg, g, ctx)
        trainer = R.Trainer(g, cfg.cameras, targets, ctx=ctx)
    tcfg = R.TrainConfig()
    lcfg = R.LossConfig(0.2)
    from rgsplat_b200 import dp

    # warm-up steps take the first view sets; every timed run (batched, plain,
    # end to end) cycles through the same args.steps view sets after them
    schedule, timed_views = view_schedule(len(cfg.cameras), V, args.warmup, args.steps, rank)
    it = iter(schedule)

    def next_views():
        try:
            return next(it)
        except StopIteration:
            v = timed_views[next_views.k % len(timed_views)]
            next_views.k += 1
            return v

    next_views.k = 0

    # multi-GPU: render + backward per rank, NCCL all-reduce of the gradient
    # planes, the same Adam update on every rank (rgsplat_b200.dp)
    dp_batched = dp.ViewParallelStep(trainer, device=f"cuda:{local_rank}", mode=R.Trainer.BATCHED) if world > 1 else None
    dp_plain = dp.ViewParallelStep(trainer, device=f"cuda:{local_rank}", mode=R.Trainer.PLAIN) if world > 1 else None

    def step_batched():
        views = next_views()
        if world == 1:
            return trainer.step(views, mode=R.Trainer.BATCHED, loss_cfg=lcfg, train_cfg=tcfg)
        return dp_batched(views, lcfg, tcfg)

    def step_plain():
        views = next_views()
        if world == 1:
            return trainer.step(views, mode=R.Trainer.PLAIN, loss_cfg=lcfg, train_cfg=tcfg)
        return dp_plain(views, lcfg, tcfg)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(fn, k: int) -> float:
        """Seconds for k steps: CUDA events on the library's stream, max over ranks.
        The steps sit in an NVTX range named after fn, so a profiler can select
        exactly the timed launches (ncu --nvtx --nvtx-include "step_batched/")."""
        barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push(fn.__name__)
            e0.record(stream)
            for _ in range(k):
                fn()
            e1.record(stream)
            torch.cuda.nvtx.range_pop()
        e1.synchronize()
        barrier()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        if dist is not None:
            tt = torch.tensor([t], device=f"cuda:{local_rank}")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    # autotuner: every blend layout timed on the first step's views (results
    # are identical across layouts), fastest kept
    tune = None
    if not args.no_autotune:
        with torch.cuda.stream(stream):
            pick, table = trainer.autotune(schedule[0], loss_cfg=lcfg, reps=2)
        tune = {"chosen": pick, "candidates_ms": table, "measured_on": "render + backward of the first step's views, mean of 2"}
    opts = ctx.options()
    layout = (f"{opts['tile_w']}x{opts['tile_h']}", opts["batch"], opts["pixels_per_thread"])

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_batched()
        ctx.set_profiling(True)
        ctx.stage_times(reset=True)
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_batched = timed(step_batched, args.steps)
    clock_info = clocks.stop()
    stage_ms = ctx.stage_times(reset=True)
    ctx.set_profiling(False)

    kp = args.plain_steps if args.plain_steps is not None else max(3, args.steps // 2)
    with torch.cuda.stream(stream):
        step_plain()
    next_views.k = 0
    t_plain = timed(step_plain, kp)

    # e2e: the step's inputs (8 RGBA targets + cameras) copied from pinned host
    # memory through the C ABI every step, losses read back.
    e2e = None
    if not args.no_e2e:
        pinned = {}

        def pinned_target(v):
            if v not in pinned:
                t = torch.from_numpy(targets[v]).pin_memory()
                pinned[v] = t
            return pinned[v]

        h2d = [0, 0]  # bytes copied host -> device, steps

        def step_e2e():
            # the same view sets as the timed batched steps, so the two numbers
            # cover the same pixels and pairs
            views = timed_views[step_e2e.k % len(timed_views)]
            step_e2e.k += 1
            ts = [pinned_target(v) for v in views]
            h2d[0] += sum(t.numel() * 4 for t in ts) + len(views) * 100
            h2d[1] += 1
            if world == 1:
                # targets copied from pinned host memory inside the step,
                # overlapped with projection, sort and forward
                return trainer.step_host_targets(views, [t.data_ptr() for t in ts], loss_cfg=lcfg, train_cfg=tcfg)
            for v, t in zip(views, ts):
                trainer.set_target_ptr(v, t.data_ptr())
            return dp_batched(views, lcfg, tcfg)

        step_e2e.k = 0
        for v in set(x for vs in timed_views for x in vs):
            pinned_target(v)
        with torch.cuda.stream(stream):
            step_e2e()
        ke = max(3, args.steps // 2)
        h2d[0] = h2d[1] = 0
        t_e2e = timed(step_e2e, ke)
        # mean over the timed steps (view sets of different resolutions)
        e2e = {"value": world * ke / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d[0] / max(h2d[1], 1)),
               "d2h_bytes_per_step": 4 * V + 8}

    value = world * args.steps / t_batched
    plain_value = world * kp / t_plain
    ms_per_step = t_batched / args.steps * 1e3

    # work per step, averaged over the timed view sets: one untimed batched
    # render + backward (no Adam) per set after the timed runs, reading the
    # pass's pair / visible-slot counts and the (pixel, splat) pairs the blend
    # kernels evaluated (rgs_trainer_evaluated_pairs)
    work = {"pairs": [], "visible": [], "entries": [], "eval_fwd": [], "eval_bwd": []}
    with torch.cuda.stream(stream):
        for vs in timed_views:
            trainer.backward(vs, loss_cfg=lcfg, mode=R.Trainer.BATCHED)
            st_w = ctx.stats()
            ef, eb = trainer.evaluated_pairs()
            work["pairs"].append(st_w["pairs"])
            work["visible"].append(st_w["visible"])
            work["entries"].append(st_w["supertile_entries"])
            work["eval_fwd"].append(ef)
            work["eval_bwd"].append(eb)
    pairs_step = float(np.mean(work["pairs"]))
    visible_step = float(np.mean(work["visible"]))
    entries_step = float(np.mean(work["entries"]))
    eval_fwd, eval_bwd = float(np.mean(work["eval_fwd"])), float(np.mean(work["eval_bwd"]))

    # roofline of the dominant stage
    pixels_per_step = int(np.mean([sum(cfg.cameras[v].width * cfg.cameras[v].height for v in vs) for vs in timed_views]))
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured"
    if not hbm:
        hbm, peak_src = 6650.0, "fallback"
    per_step_ms = {k: v / args.steps for k, v in stage_ms.items() if v > 0}
    dom = max(per_step_ms, key=per_step_ms.get) if per_step_ms else None
    roofline = None
    stages = {}
    for k, ms in per_step_ms.items():
        b = algorithmic_bytes(k, n, V, pairs_step, pixels_per_step, visible_step, entries_step)
        gbs = b / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        stages[k] = {"ms": round(ms, 4), "algorithmic_gb": round(b / 1e9, 4), "achieved_gbs": round(gbs, 1), "frac_hbm": round(gbs / hbm, 4)}
    # FP32 roofline of the blend kernels: evaluated (pixel, splat) pairs x the
    # reference algorithm's FP32 operations per pair (forward ~20 + one exp,
    # backward ~45 + one exp + one divide; FMA counted as 2), against
    # SMs x 128 FP32 lanes x 2 x the median SM clock sampled while timing
    props = torch.cuda.get_device_properties(local_rank)
    clock_mhz = clock_info.get("sm_mhz") or clock_info.get("sm_max_mhz") or 1965.0
    fp32_peak = props.multi_processor_count * 128 * 2 * clock_mhz * 1e6 / 1e12
    fp32 = {}
    for k, pairs_eval, fpp in (("forward", eval_fwd, 20), ("backward", eval_bwd, 45)):
        ms = per_step_ms.get(k)
        if not ms:
            continue
        tf = pairs_eval * fpp / (ms / 1e3) / 1e12
        fp32[k] = {"evaluated_pairs": int(pairs_eval), "flops_per_pair": fpp, "exp_per_pair": 1,
                   "achieved_tflops": round(tf, 3), "peak_tflops": round(fp32_peak, 2), "frac": round(tf / fp32_peak, 4),
                   "pairs_per_ns": round(pairs_eval / (ms * 1e6), 3)}
        stages[k]["fp32"] = fp32[k]
    if dom:
        b = algorithmic_bytes(dom, n, V, pairs_step, pixels_per_step, visible_step, entries_step)
        ach = b / (per_step_ms[dom] / 1e3) / 1e9
        traffic = profiled_traffic("blend_bwd_1M_8views.md") if dom == "backward" and args.scale == 1.0 else None
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 4), "peak_source": peak_src, "traffic": traffic,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel at this workload, "
                                      "profiles/blend_bwd_1M_8views.md" if traffic else None,
                    "algorithmic_bytes": int(b),
                    "fp32": {**fp32.get(dom, {}), "peak_source": f"{props.multi_processor_count} SMs x 128 FP32 lanes "
                                                                f"x 2 x {clock_mhz:.0f} MHz (median sampled SM clock)"},
                    "issue_active": profiled_issue_active("k_blend_bwd") if dom == "backward" else None,
                    "note": "the blend kernels are bound by instruction issue, not DRAM (issue_active: fraction of issue "
                            "slots busy, ncu, profiles/blend_pipes_250k_8views.md); fp32 is the roof that applies, "
                            "the HBM fraction is reported as the contract asks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            s_iter, iters, threads, _ = oracle_iterations(g, cfg, timed_views, lambda v: targets[v], 0.0, 1)
            cpu = {"value": 1.0 / s_iter, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{iters} whole iteration ({V} x render_and_backward + one Adam step, {s_iter:.2f} s) of "
                             f"this workload on the oracle, on the first timed view set"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config(cfg, n, V, world),
            "mode": "batched (graph-captured, one launch per stage)",
            "layout": {"tile": layout[0], "batch": layout[1], "pixels_per_thread": layout[2], "autotune": tune},
            "plain": {"value": round(plain_value, 4), "unit": UNIT, "steps": kp, "batched_over_plain": round(value / plain_value, 3)},
            "work_per_step": {"pairs": int(pairs_step), "visible_slots": int(visible_step),
                              "supertile_entries": int(entries_step), "pixels": pixels_per_step,
                              "evaluated_pairs_forward": int(eval_fwd), "evaluated_pairs_backward": int(eval_bwd),
                              "measured_on": "an untimed render + backward of each timed view set after the timed runs"},
            "e2e": e2e,
            "gpu_launches": None,
            "roofline": roofline,
            "stages": stages,
            "cpu_baseline": cpu,
            "clocks": clock_info,
        }
        if not args.no_variants:
            line["backward_variants"] = measure_backward_variants(R, scenes, local_rank)
        if not args.no_rows and world == 1:
            line["next_rows"] = measure_next_rows(R, g, cfg.cameras[0], local_rank, cpu=not args.no_cpu_baseline)
        # kernels launched per batched step (+ memsets): term cache + project 2;
        # compaction 3 (counts, scan, gather); depth sort 4 passes x 3; two
        # count scans 2 x 2; emit 1; supertile sort 3 per 8 bits of the
        # supertile id; tile lists 3 (masks, scan, writer); forward 1; loss 2;
        # backward 1; geometry + Adam 3 (per view, SH half, geometry half)
        ltw, lth = (int(x) for x in layout[0].split("x"))
        cdiv = lambda a, b: -(-a // b)
        st_view = max(cdiv(cdiv(c.width, ltw), 4) * cdiv(cdiv(c.height, lth), 4) for c in cfg.cameras)
        st_bits = max(1, int(np.ceil(np.log2(max(2, V * st_view)))))
        per_step = 2 + 3 + 12 + 4 + 1 + 3 * ((st_bits + 7) // 8) + 3 + 1 + 2 + 1 + 3
        line["gpu_launches"] = per_step * args.steps
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
