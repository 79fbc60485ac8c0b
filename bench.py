#!/usr/bin/env python
"""Points x iterations per second of the bundling loop on the large workload.

Workload: 100,000 seeded random-walk polylines (2..8 control points each),
4.95M samples at spacing 1/1000 of the canvas, 2048^2 density grid, blur
sigma 16 px, neighbour radius 16 texels (synthetic stand-in for the
reference's datasets, which are LFS stubs). A step is one bundling iteration
(Gpu::iterate: neighbour mean fused with the splat, grid rebuild, blur,
normalisation) with all data resident in HBM; the step's working set
(~330 MB) is larger than the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank runs an independent replica (the path does not
shard; scaling is weak) and rank 0 prints one JSON line. `--impl reference`
times the CPU restatement of the reference's algorithm (the reference itself
is Rust + wgpu and cannot run here) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points·iter/s at 100k edges"
UNIT = "points·iter/s"
ITERATIONS_PER_JOB = 30
# Algorithmic bytes per sample of the fused neighbour-mean kernel: read
# position record 8 + tag 4; write position 8 + tag 4 + next search cell 4;
# population atomic 4 + splat atomic 4.
MEAN_BYTES_PER_SAMPLE = 36


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10, help="large workload: timed jobs (30 iterations each)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--edges", type=int, default=100_000)
    p.add_argument("--e2e-jobs", type=int, default=3)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU work of the baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", choices=["large", "batched", "served", "render", "advect"], default="large")
    p.add_argument("--advect-step", type=float, default=1.0, help="advect workload: texels per iteration")
    p.add_argument("--advect-smooth", type=float, default=0.5, help="advect workload: path relaxation weight")
    p.add_argument("--render-iterations", type=int, default=30,
                   help="render workload: mean updates before the frames are drawn")
    p.add_argument("--steady-iterations", type=int, default=200,
                   help="large workload: iterations of the steady-state figure past the job (0 = skip)")
    p.add_argument("--quick", action="store_true", help="large workload only: no e2e, batched, served or CPU legs")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-served", action="store_true")
    p.add_argument("--graphs", type=int, default=256, help="batched workload: number of graphs")
    p.add_argument("--batch-iterations", type=int, default=10)
    p.add_argument("--requests", type=int, default=1000, help="served workload: requests per rank")
    p.add_argument("--rate", type=float, default=200.0, help="served workload: mean arrivals per second")
    p.add_argument("--capacity-requests", type=int, default=200,
                   help="served: requests of the all-at-once capacity run")
    p.add_argument("--latency-requests", type=int, default=150,
                   help="served: requests of each latency run at a fraction of the plain loop's capacity")
    p.add_argument("--latency-fractions", type=float, nargs="*", default=[0.5, 0.8, 1.0])
    p.add_argument("--solo-samples", type=int, default=0,
                   help="served: requests of at least this many samples iterate beside the batch (0 = 32768)")
    p.add_argument("--max-active", type=int, default=32)
    p.add_argument("--max-step", type=int, default=1)
    p.add_argument("--budget-gb", type=float, default=120.0)
    p.add_argument("--reserve-gb", type=float, default=48.0, help="served workload: device memory mapped at start")
    return p.parse_args(argv)


def pinned_buffer(nbytes: int) -> np.ndarray:
    """Page-locked host bytes (read-backs into them run at full PCIe speed)."""
    import torch

    return torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()


# ---------------------------------------------------------------- ranks
class Ranks:
    def __init__(self, want: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist
            self.torch = torch
            self.backend = backend

    def _t(self, x):
        t = self.torch.tensor([float(x)], dtype=self.torch.float64)
        return t.cuda() if self.backend == "nccl" else t

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        t = self._t(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return x
        t = self._t(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.first = threading.Event()

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def wait_first(self, timeout: float = 5.0) -> None:
        """Block until nvidia-smi has printed its first sample, so that the
        timed region that follows is covered from its start."""
        if self.proc:
            self.first.wait(timeout)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum: 99.60 + 49.79 MB)
# of one launch of the neighbour-mean kernel on the large workload, iteration
# 15 of a job, from one ncu capture (1 pass) of this kernel on B200:
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum \
#       --clock-control none -k regex:neighbor_mean -s 14 -c 1 \
#       python bench.py --quick --steps 1 --warmup 0 --steady-iterations 0
MEAN_TRAFFIC_BYTES = 149_390_000


def workload(edges: int):
    from bundling_thingy_b200 import synthetic

    return synthetic.large(edges)


# ---------------------------------------------------------------- CPU sample
def cpu_sample(w, target_seconds: float, steps: int = 1, warmup: int = 0, threads: int = 0):
    """Bounded CPU timing of the oracle (the reference's algorithm restated):
    neighbour mean of every s-th sample (s chosen so one step is about
    target_seconds) plus a full density pass charged pro rata."""
    import oracle as O

    threads = threads or len(os.sched_getaffinity(0))
    cfg = O.Config(w.width, w.height, radius=w.radius, resample_scale=(500.0, 500.0),
                   sigma=float(np.float32(w.sigma)), threads=threads)
    pipe = O.Pipeline(cfg)
    n = pipe.upload(w.xy, w.starts)
    xy, _ = pipe.points()
    mv = O.movable_mask(pipe.paths(), n)
    taps = O.blur_weights(float(np.float32(w.sigma)))
    # Calibrate the stride on a small probe (query time only).
    probe = max(1, n // 2000)
    _, done, t_index, t_call = O.neighbor_mean_sample(xy, mv, w.width, w.height, w.radius, probe, threads)
    per_sample = max(t_call - t_index, 1e-9) / max(done, 1)
    stride = max(1, int(np.ceil(n * per_sample / target_seconds)))
    sampled = (n + stride - 1) // stride
    values = []
    for i in range(warmup + steps):
        out, done, t_index, t_call = O.neighbor_mean_sample(xy, mv, w.width, w.height, w.radius, stride, threads)
        t_query = max(t_call - t_index, 0.0)
        t0 = time.perf_counter()
        counts = O.splat(out, w.width, w.height)
        _, vt, peak = O.blur(counts, w.width, w.height, taps)
        O.normalize(vt, peak)
        t_density = time.perf_counter() - t0
        # The sampled samples over their query time plus the whole-set grid
        # index and density pass charged for their share of the samples.
        share = sampled / n
        if i >= warmup:
            values.append(sampled / (t_query + (t_index + t_density) * share))
    return {
        "value": float(statistics.median(values)),
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": (f"neighbour mean of the first {sampled} of {n} samples (whole paths) of the large workload "
                   f"+ the whole-set grid index and density pass charged pro rata, "
                   f"{steps} step(s), OpenMP over {threads} host threads"),
    }


# ---------------------------------------------------------------- reference arm
def run_reference(args, ranks: Ranks):
    if ranks.rank != 0:
        return
    w = workload(args.edges)
    # Each step is a bounded sample: about two minutes of neighbour-mean work
    # over the whole run (at most 2 s and at least 0.25 s a step), so that the
    # default 200 + 10 steps end within a few minutes; each step also repeats
    # the whole-set grid index and density pass (about 0.2 s on 16 threads).
    target = min(2.0, max(0.25, 120.0 / max(1, args.steps + args.warmup)))
    base = cpu_sample(w, target_seconds=target, steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference",
        "metric": METRIC, "value": base["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random-walk polylines; reference datasets are LFS stubs)",
        "config": {"workload": "large: 100k polylines, 4.95M samples, 2048^2, sigma 16, radius 16",
                   "iterations_per_job": ITERATIONS_PER_JOB},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference is Rust + wgpu/Vulkan (no rustc, no graphics stack on this box); "
                 "its algorithm is timed through the CPU restatement in oracle/"),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
# Kernels per iteration: neighbour mean, cell table (tile-sum scan + apply),
# scatter, slot prefix (reduce + tile-sum scan + apply) on the context's
# stream; blur H, blur V + maximum, normalise beside them.
KERNELS_PER_ITERATION = 10


def pinned_copy(a):
    t = pinned_buffer(a.nbytes).view(a.dtype).reshape(a.shape)
    t[...] = a
    return t


def run_ours(args, ranks: Ranks):
    """The configured job on the large workload: upload, then 30 iterations
    (Gpu::iterate), timed with CUDA events on the library's stream from the
    first iteration after the upload to the last. A step is one such job; the
    upload that resets the geometry before each step is not timed (its device
    inputs are then resident). The steady state past the job, the stage
    split, the end-to-end job through host buffers, the batched and served
    workloads and the CPU baseline are reported beside it."""
    import bundling_thingy_b200 as bt

    w = workload(args.edges)
    device = ranks.local
    iters = ITERATIONS_PER_JOB
    opts = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                      blur_sigma=w.sigma, device=device)
    gpu = bt.Gpu(opts)
    sampler = ClockSampler(device)
    sampler.start()
    sampler.wait_first()
    n = 0
    for _ in range(args.warmup):
        n = gpu.upload((w.xy, w.starts))
        gpu.iterate(iters)
    job_ms = []
    ranks.barrier()
    gpu.synchronize()
    for _ in range(args.steps):
        n = gpu.upload((w.xy, w.starts))
        job_ms.append(gpu.iterate_timed(iters))
    gpu.synchronize()
    ranks.barrier()
    clocks = sampler.stop()
    info = gpu.info()
    ms_max = ranks.max(sum(job_ms))
    value = ranks.sum(float(n) * iters * args.steps) / (ms_max / 1e3)

    # Steady state past the job: 10 more iterations, then the timed ones.
    steady_ms = None
    if args.steady_iterations:
        gpu.iterate(10)
        steady_ms = ranks.max(gpu.iterate_timed(args.steady_iterations))
    gpu.close()

    # The same jobs with the search-shape checks option (off by default).
    checks_ms = checks_value = None
    if args.steps:
        chk = bt.Gpu(bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                                blur_sigma=w.sigma, device=device, shape_checks=True))
        chk.upload((w.xy, w.starts))
        chk.iterate(iters)
        ranks.barrier()
        jobs = []
        for _ in range(min(args.steps, 5)):
            chk.upload((w.xy, w.starts))
            jobs.append(chk.iterate_timed(iters))
        chk.close()
        checks_ms = ranks.max(sum(jobs) / len(jobs))
        checks_value = ranks.sum(float(n) * iters) / (checks_ms / 1e3)

    # Stage split of one job (per-stage CUDA events; the iterations run as
    # direct launches instead of a CUDA graph): iteration 1 alone, then 2-30.
    st = bt.Gpu(bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                           blur_sigma=w.sigma, device=device, timing=True))
    st.upload((w.xy, w.starts))
    st.iterate(1)
    first = st.stage_times()
    st.iterate(iters - 1)
    rest = st.stage_times()
    st.close()
    stages = {k: first.get(k, 0.0) + rest.get(k, 0.0) for k in set(first) | set(rest)}
    stages = dict(sorted(stages.items(), key=lambda kv: -kv[1]))
    total_stage = sum(stages.values())
    mean_ms = stages.get("graph.neighbor_mean", float("nan")) / iters
    peak, peak_kind = measured_peak_hbm()
    bytes_per_launch = MEAN_BYTES_PER_SAMPLE * n
    achieved = bytes_per_launch / (mean_ms / 1e3) / 1e9

    # End to end through the public API with host buffers: upload the control
    # points, 30 iterations, read back the 12-byte records and the density.
    e2e_value = job = None
    h2d = d2h = 0
    if args.e2e_jobs > 0:
        e2e_gpu = bt.Gpu(opts)
        xy_h, starts_h = pinned_copy(w.xy), pinned_copy(w.starts)
        records = pinned_buffer(12 * n)
        dens = pinned_buffer(w.width * w.height * 4).view(np.float32)
        job_times = []
        for j in range(args.e2e_jobs + 1):
            ranks.barrier()
            t0 = time.perf_counter()
            e2e_gpu.upload((xy_h, starts_h))
            e2e_gpu.iterate(iters)
            e2e_gpu.read_records(records)
            e2e_gpu.read_density(dens)
            t = time.perf_counter() - t0
            if j > 0:  # the first job warms host paths
                job_times.append(t)
        e2e_gpu.close()
        job = ranks.max(statistics.median(job_times))
        e2e_value = ranks.sum(float(n) * iters) / job
        h2d = w.xy.nbytes + w.starts.nbytes
        d2h = records.nbytes + dens.nbytes

    batched = batched_measure(args, ranks) if not args.no_batched else None
    served = served_measure(args, ranks) if not args.no_served else None

    cpu = None
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(w, target_seconds=args.cpu_seconds)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random-walk polylines; reference datasets are LFS stubs)",
        "config": {
            "workload": "large: 100k polylines (2-8 control points), 2048^2, spacing 1/1000, sigma 16 px, radius 16",
            "step": f"one job: iterations 1-{iters} after an upload (the upload before each step is not timed)",
            "samples": n, "edges": w.edges, "grid": [w.width, w.height], "radius": w.radius, "sigma": w.sigma,
            "search_cells_per_grid_cell": {"x": info.fine_cells_x, "y": info.fine_cells,
                                           "chosen": "at upload from the graph's density"},
            "iterations_per_job": iters,
            "parallelism": f"replicas x{ranks.world}", "l2": "inputs larger than L2 (~330 MB working set per step)",
        },
        "ms_per_iteration": ms_max / args.steps / iters,
        "shape_checks_option": None if checks_ms is None else {
            "value": checks_value, "unit": UNIT, "ms_per_job": checks_ms,
            "note": "same jobs with options.shape_checks = 1 (off by default: 4% faster here, slower on "
                    "small-radius graphs)"},
        "steady_state": None if steady_ms is None else {
            "value": ranks.sum(float(n) * args.steady_iterations) / (steady_ms / 1e3), "unit": UNIT,
            "ms_per_iteration": steady_ms / args.steady_iterations,
            "iterations": f"{iters + 11}-{iters + 10 + args.steady_iterations} after the upload"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "step": f"upload + {iters} iterations + readback of records and density",
                "seconds_per_job": job},
        "roofline": {
            "kernel": "neighbor_mean", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": MEAN_TRAFFIC_BYTES if args.edges == 100_000 else None,
            "peak_source": peak_kind,
            "bytes_per_launch": bytes_per_launch, "ms_per_launch": mean_ms,
            "launches": f"iterations 1-{iters} of one job",
            "ms_iteration_1": first.get("graph.neighbor_mean"),
            "note": "issue-bound: the exact test of each sample's boundary band at radius 16",
        },
        "stage_ms_per_iteration": {k: v / iters for k, v in stages.items()},
        "stage_share": {k: v / total_stage for k, v in stages.items()} if total_stage else {},
        "gpu_launches": KERNELS_PER_ITERATION * iters * args.steps,
        "clocks": clocks,
        "batched": batched,
        "served": served,
        "cpu_baseline": cpu,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- render
def run_render(args, ranks: Ranks):
    """Frames of the large workload's bundled geometry (bt_render: tile
    binning, ordered blending, endpoint-free density colouring at 4x MSAA,
    the reference's render defaults), against the oracle's rasteriser on one
    host thread."""
    import bundling_thingy_b200 as bt

    w = workload(args.edges)
    device = ranks.local
    opts = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                      blur_sigma=w.sigma, device=device)
    gpu = bt.Gpu(opts)
    n = gpu.upload((w.xy, w.starts))
    gpu.iterate(args.render_iterations)
    segments = gpu.info().segments
    for _ in range(max(args.warmup, 3)):
        gpu.render(pixels=False)
    sampler = ClockSampler(device)
    sampler.start()
    ranks.barrier()
    frame_ms = [gpu.render(pixels=False).device_ms for _ in range(args.steps)]
    ranks.barrier()
    clocks = sampler.stop()
    ms = ranks.max(statistics.median(frame_ms))
    value = ranks.sum(1.0) / (ms / 1e3)
    # End to end: the frame and its RGBA8 readback into pinned host memory.
    import torch

    rgba = torch.empty(w.width * w.height * 4, dtype=torch.uint8, pin_memory=True).numpy().reshape(
        w.height, w.width, 4)
    walls = []
    for i in range(args.steps + 1):
        t0 = time.perf_counter()
        f = gpu.render(out=rgba)
        if i:
            walls.append(time.perf_counter() - t0)
    wall = ranks.max(statistics.median(walls))
    colored = f.colored_pixels
    cpu = None
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        import oracle as O

        xy, ids = gpu.read_points()
        seg, paths, dens = gpu.read_segments(), gpu.read_paths(), gpu.read_density()
        t0 = time.perf_counter()
        _, c_colored = O.render(xy, ids, seg, paths.shape[0], dens, w.width, w.height)
        t_cpu = time.perf_counter() - t0
        assert c_colored == colored
        cpu = {"value": 1.0 / t_cpu, "unit": "frames/s", "cores": 1, "kind": "port",
               "sample": f"one whole frame ({segments} segments, {w.width}x{w.height}, 4x MSAA) by the oracle's "
                         f"sequential rasteriser; same coloured-pixel count"}
    gpu.close()
    line = {
        "metric": "frames/s", "value": value, "unit": "frames/s", "n_gpus": ranks.world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/i64",
        "data": "synthetic (seeded random-walk polylines)",
        "config": {"workload": (f"render: large ({n} samples, {segments} segments) after "
                                f"{args.render_iterations} iterations, {w.width}x{w.height}, 4x MSAA, density "
                                "colour, no endpoint dots"),
                   "colored_pixels": colored, "l2": "frame state (64 MB of samples) rewritten each frame"},
        "e2e": {"value": 1.0 / wall, "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": w.width * w.height * 4 + 16,
                "step": "bt_render with the RGBA8 readback into pinned host memory"},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- advect
def run_advect(args, ranks: Ranks):
    """Iterations of the density-gradient advection mode (an extension beyond
    the reference) on the large workload, against the oracle's step with its
    splat, blur and normalisation on all host threads."""
    import bundling_thingy_b200 as bt

    w = workload(args.edges)
    device = ranks.local
    opts = bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma, device=device,
                      advect_step=args.advect_step, advect_smooth=args.advect_smooth)
    gpu = bt.Gpu(opts)
    n = gpu.upload((w.xy, w.starts))
    gpu.iterate(max(args.warmup, 3))
    sampler = ClockSampler(device)
    sampler.start()
    ranks.barrier()
    ms = gpu.iterate_timed(args.steps)
    ranks.barrier()
    clocks = sampler.stop()
    ms_max = ranks.max(ms)
    value = ranks.sum(float(n) * args.steps) / (ms_max / 1e3)
    cpu = None
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        import oracle as O

        xy, ids = gpu.read_points()
        dens = gpu.read_density()
        taps = O.blur_weights(float(np.float32(w.sigma)))
        t0 = time.perf_counter()
        out = O.advect(xy, ids, dens, w.width, w.height, args.advect_step, args.advect_smooth)
        counts = O.splat(out, w.width, w.height)
        _, vt, peak = O.blur(counts, w.width, w.height, taps)
        O.normalize(vt, peak)
        t_cpu = time.perf_counter() - t0
        threads = len(os.sched_getaffinity(0))
        cpu = {"value": n / t_cpu, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one whole iteration ({n} samples): advection step with OpenMP over {threads} host "
                         f"threads, splat, blur and normalisation"}
    gpu.close()
    line = {
        "metric": METRIC.replace("at 100k edges", "at 100k edges, advection mode"), "value": value, "unit": UNIT,
        "n_gpus": ranks.world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random-walk polylines)",
        "config": {"workload": (f"advect: large ({n} samples, 2048^2, sigma {w.sigma}), step "
                                f"{args.advect_step} texels, smoothing {args.advect_smooth}"),
                   "l2": "inputs larger than L2"},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- sharding
def shard(items, ranks: Ranks):
    """The graphs one rank bundles: every world-th item from its rank (the
    batched workload's graphs are independent; no collective)."""
    return list(items)[ranks.rank::ranks.world]


def served_seed(rank: int) -> int:
    """Seed of a rank's own arrival stream (and its graphs) in the served
    workload; rank 0 replays the workload's own seed."""
    from bundling_thingy_b200 import synthetic

    return synthetic.SEED_BASE + 4 + 7919 * rank


# ---------------------------------------------------------------- batched
def batched_measure(args, ranks: Ranks) -> dict:
    """256 independent graphs (edges log-uniform 200-20,000, grids 256/512/1024),
    10 iterations each: one batch (persistent launches over graph x tile,
    CUDA-graph iteration) against the plain per-graph loop. Graphs are
    sharded across ranks by index (no collective)."""
    import bundling_thingy_b200 as bt
    from bundling_thingy_b200 import synthetic

    device = ranks.local
    iters = args.batch_iterations
    jobs = shard(synthetic.batched_jobs(args.graphs, iterations=iters), ranks)

    def key(j):
        return (j.width, j.radius)

    def options(j):
        return bt.Options(width=j.width, height=j.height, neighbor_radius=j.radius, sample_spacing=j.spacing,
                          blur_sigma=j.sigma, device=device)

    # Plain per-graph loop: one context per class, reused (Gpu::upload
    # releases the previous graph), upload + 10 x iterate + readback.
    # Results are read into one reused pinned host buffer in both arms.
    host = {"buf": None}

    def read(g):
        n = 12 * g.info().samples
        if host["buf"] is None or host["buf"].nbytes < n:
            host["buf"] = pinned_buffer(max(n, 96 << 20))
        return g.read_records(host["buf"])

    # Warm-up of both arms to their steady state: each reused context holds
    # the buffers of its class's largest graph, and the device memory pool
    # has mapped the memory of a whole batch once.
    largest = {}
    for j in jobs:
        if key(j) not in largest or j.starts.size > largest[key(j)].starts.size:
            largest[key(j)] = j
    ctxs = {k: bt.Gpu(options(j)) for k, j in largest.items()}
    for k, j in largest.items():
        ctxs[k].upload((j.xy, j.starts))
        ctxs[k].iterate(1)
        read(ctxs[k])
    ranks.barrier()
    plain_results = {}
    t0 = time.perf_counter()
    t_iter = 0.0
    for idx, j in enumerate(jobs):
        g = ctxs[key(j)]
        g.upload((j.xy, j.starts))
        ti = time.perf_counter()
        g.iterate(iters)
        t_iter += time.perf_counter() - ti
        rec = read(g)
        if idx < 4:
            plain_results[idx] = rec.copy()
    plain_s = time.perf_counter() - t0
    for g in ctxs.values():
        g.close()

    # The batch's work shape from the autotuner (scratch batches of the same
    # graphs, outside the timed region).
    shape, _ = bt.Batch.autotune([(options(j), j.xy, j.starts) for j in jobs], iterations=iters, device=device)

    # Warm the batch kernels once (module load, first graph capture).
    warm = bt.Batch(device)
    warm.set_shape(**shape)
    warm.add_many([(options(j), j.xy, j.starts) for j in jobs])
    warm.iterate(1)
    warm.close()

    # Batched: upload every graph concurrently, one batched call for all
    # iterations, readback.
    ranks.barrier()
    t0 = time.perf_counter()
    batch = bt.Batch(device)
    batch.set_shape(**shape)
    slots = [s for s, _ in batch.add_many([(options(j), j.xy, j.starts) for j in jobs])]
    t_add = time.perf_counter() - t0
    ti = time.perf_counter()
    batch.iterate(iters)
    batch_iter_s = time.perf_counter() - ti
    outs = {}
    for idx, s in enumerate(slots):
        rec = read(batch.slot(s))
        if idx < 4:
            outs[idx] = rec.copy()
    batch_s = time.perf_counter() - t0
    exact = all(np.array_equal(outs[i], plain_results[i]) for i in plain_results)
    samples = sum(batch.slot(s).info().samples for s in slots)
    # Device time of the batched iterations alone (CUDA events).
    dev_ms = batch.iterate_timed(iters)
    batch.close()

    graphs = ranks.sum(len(jobs))
    batch_gps = graphs / ranks.max(batch_s)
    plain_gps = graphs / ranks.max(plain_s)
    return {
        "graphs_per_s": batch_gps, "plain_graphs_per_s": plain_gps, "speedup_vs_plain": batch_gps / plain_gps,
        "iteration_speedup_vs_plain": ranks.sum(t_iter) / ranks.sum(batch_iter_s),
        "batch_seconds": {"add_uploads": t_add, "iterations": batch_iter_s, "total": batch_s},
        "plain_seconds": {"iterations": t_iter, "total": plain_s},
        "device_points_iter_per_s": ranks.sum(samples * iters) / (ranks.max(dev_ms) / 1e3),
        "graphs": int(graphs), "samples": int(ranks.sum(samples)), "iterations": iters,
        "tuned_shape": shape,
        "search_cells": "chosen per graph at upload from its density",
        "bit_exact_vs_plain": exact,
        "step": "upload + iterations + pinned readback of every graph, both arms warmed first",
    }


def run_batched(args, ranks: Ranks):
    m = batched_measure(args, ranks)
    line = {
        "metric": f"batched graphs/s ({args.graphs} graphs, {args.batch_iterations} iterations each)",
        "value": m["graphs_per_s"], "unit": "graphs/s", "n_gpus": ranks.world, "higher_is_better": True,
        "scaling": "weak", "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched: 256 graphs, edges log-uniform 200-20k, grids 256/512/1024, 10 iterations",
                   "parallelism": f"graphs sharded x{ranks.world}"},
        **m,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- served
class ServedBench:
    """Poisson-arriving requests (edges log-uniform 500-50,000; grids
    512/1024/2048; 10 iterations each; 120 GB admission budget): the
    continuous-batching server against the plain per-request loop, both
    replaying the same arrival schedule and reading every result back to
    pinned host memory. Each rank serves its own arrival stream (weak
    scaling, no collective)."""

    keep = 4   # results compared between the arms

    def __init__(self, args, ranks: Ranks, requests: int):
        import bundling_thingy_b200 as bt
        from bundling_thingy_b200 import synthetic

        self.bt, self.args, self.ranks = bt, args, ranks
        self.device = ranks.local
        self.iters = args.batch_iterations
        self.arrivals, self.jobs = synthetic.served_jobs(requests, rate=args.rate, iterations=self.iters,
                                                         seed=served_seed(ranks.rank))
        self.largest = {}  # (grid, radius) class -> index of its largest request
        for i, j in enumerate(self.jobs):
            k = self.key(j)
            if k not in self.largest or j.starts.size > self.jobs[self.largest[k]].starts.size:
                self.largest[k] = i
        by_size = sorted(range(len(self.jobs)), key=lambda i: -self.jobs[i].starts.size)
        self.warm_set = by_size[: max(len(self.largest), args.max_active)]
        self.opts = [bt.Options(width=j.width, height=j.height, neighbor_radius=j.radius, sample_spacing=j.spacing,
                                blur_sigma=j.sigma, device=self.device) for j in self.jobs]
        self.host = None

    @staticmethod
    def key(j):
        return (j.width, j.radius)

    def pinned(self, nbytes):
        if self.host is None or self.host.nbytes < nbytes:
            self.host = pinned_buffer(max(nbytes, 128 << 20))
        return self.host

    def plain(self, sched):
        """Plain per-request loop: one reused context per (grid, radius)
        class; upload, 10 iterations, read back, in arrival order."""
        bt, jobs = self.bt, self.jobs
        ctxs = {}
        for k, i in self.largest.items():      # each context sized for its class's largest graph
            j = jobs[i]
            g = bt.Gpu(self.opts[i])
            g.upload((j.xy, j.starts))
            g.iterate(1)
            g.read_records(self.pinned(12 * g.info().samples))
            ctxs[k] = g
        lat, kept, samples = [], {}, 0
        base = time.perf_counter() + 0.05
        t_end = base
        for i, (a, j) in enumerate(zip(sched, jobs[: len(sched)])):
            target = base + a
            wait = target - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            g = ctxs[self.key(j)]
            nsamp = g.upload((j.xy, j.starts))
            g.iterate(self.iters)
            rec = g.read_records(self.pinned(12 * nsamp))
            t_end = time.perf_counter()
            lat.append(t_end - target)
            samples += nsamp
            if i < self.keep:
                kept[i] = rec.copy()
        for g in ctxs.values():
            g.close()
        return {"lat": lat, "span": t_end - (base + sched[0]), "samples": samples, "kept": kept}

    def served(self, sched):
        args, jobs = self.args, self.jobs
        server = self.bt.Server(self.device, max_active=args.max_active, budget_bytes=int(args.budget_gb * 1e9),
                                max_step=args.max_step, reserve_bytes=int(args.reserve_gb * 1e9),
                                solo_samples=args.solo_samples)
        # Warm-up to the steady state: the max_active largest requests at
        # once (kernels, device memory pool, idle contexts sized for large
        # graphs, like the plain loop's reused contexts).
        for i in self.warm_set:
            server.submit(self.opts[i], jobs[i].xy, jobs[i].starts, 1)
        for _ in self.warm_set:
            r = server.next(120.0)
            server.read_records(r.id, r.samples, self.pinned(12 * r.samples))
            server.release(r.id)
        t0 = time.perf_counter()
        base = server.clock() + 1.0 + 2e-3 * len(sched)   # after every submission
        ids = {}
        for i, (a, j) in enumerate(zip(sched, jobs[: len(sched)])):
            ids[server.submit(self.opts[i], j.xy, j.starts, self.iters, arrival_s=base + a)] = i
        submit_s = time.perf_counter() - t0
        late = server.clock() > base
        lat, kept, samples, t_end = [], {}, 0, base
        for _ in range(len(sched)):
            r = server.next(300.0)
            if r.status != 0:
                raise RuntimeError(f"request {r.id} failed: {r.message}")
            rec = server.read_records(r.id, r.samples, self.pinned(12 * r.samples))
            t_end = server.clock()
            lat.append(t_end - r.arrival_s)
            samples += r.samples
            if ids[r.id] < self.keep:
                kept[ids[r.id]] = rec.copy()
            server.release(r.id)
        stats = server.stats()
        server.close()
        return {"lat": lat, "span": t_end - (base + sched[0]), "samples": samples, "kept": kept, "stats": stats,
                "submit_s": submit_s, "late": late}

    def both(self, sched):
        self.ranks.barrier()
        s = self.served(sched)
        self.ranks.barrier()
        p = self.plain(sched)
        s["exact"] = s["samples"] == p["samples"] and all(np.array_equal(s["kept"][i], p["kept"][i])
                                                         for i in p["kept"])
        return s, p

    def rate(self, m, span):
        return self.ranks.sum(m / self.ranks.max(span))


def pct(lat):
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "max_ms": float(np.max(lat) * 1e3)}


def served_measure(args, ranks: Ranks) -> dict:
    """Capacity of both arms (every request arrives at once), then p50/p99
    latency of both arms at fixed fractions of the plain loop's capacity,
    replaying the same Poisson draws on a slower or faster clock."""
    sb = ServedBench(args, ranks, max(args.capacity_requests, args.latency_requests))
    m = min(args.capacity_requests, len(sb.jobs))
    cs, cp = sb.both(np.zeros(m))
    cap_s, cap_p = sb.rate(m, cs["span"]), sb.rate(m, cp["span"])
    out = {
        "capacity": {"requests": m, "served_graphs_per_s": cap_s, "plain_graphs_per_s": cap_p,
                     "speedup_vs_plain": cap_s / cap_p, "bit_exact_vs_plain": cs["exact"],
                     "served_peak_active": cs["stats"]["peak_active"]},
        "latency": [],
        "config": {"iterations": sb.iters, "max_active": args.max_active, "max_step": args.max_step,
                   "solo_samples": args.solo_samples or 32768, "budget_gb": args.budget_gb,
                   "edges": "log-uniform 500-50k", "grids": "512/1024/2048"},
    }
    m = min(args.latency_requests, len(sb.jobs))
    unit = np.asarray(sb.arrivals[:m]) * args.rate    # Poisson draws at one arrival per unit
    for frac in args.latency_fractions:
        rate = frac * cap_p / max(ranks.world, 1)     # per rank, against the plain loop's capacity
        ls, lp = sb.both(unit / rate)
        out["latency"].append({
            "fraction_of_plain_capacity": frac, "rate_per_s": rate, "requests": m,
            "served": pct(ls["lat"]), "plain": pct(lp["lat"]),
            "served_graphs_per_s": sb.rate(m, ls["span"]), "plain_graphs_per_s": sb.rate(m, lp["span"]),
            "bit_exact_vs_plain": ls["exact"]})
    return out


def run_served(args, ranks: Ranks):
    """The served workload at its configured rate (Poisson 200/s) plus the
    capacity and latency figures of served_measure."""
    sb = ServedBench(args, ranks, args.requests)
    clocks = ClockSampler(ranks.local)
    clocks.start()
    clocks.wait_first()
    s, p = sb.both(sb.arrivals)
    clock_info = clocks.stop()
    n = len(sb.jobs)
    served_gps, plain_gps = sb.rate(n, s["span"]), sb.rate(n, p["span"])
    stats = s["stats"]
    line = {
        "metric": f"served graphs/s (Poisson {args.rate:g}/s, {sb.iters} iterations each)", "value": served_gps,
        "unit": "graphs/s", "n_gpus": ranks.world, "higher_is_better": True, "scaling": "weak", "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"served: {n} Poisson requests per rank at {args.rate:g}/s, edges log-uniform "
                               f"500-50k, grids 512/1024/2048, {sb.iters} iterations, "
                               f"{args.budget_gb:g} GB admission budget",
                   "max_active": args.max_active, "max_step": args.max_step, "reserve_gb": args.reserve_gb,
                   "solo_samples": args.solo_samples or 32768,
                   "warm": "both arms warmed with the largest graphs first (device memory pool mapped, "
                           "contexts sized); inputs larger than L2",
                   "parallelism": f"one arrival stream per rank x{ranks.world}"},
        "latency": pct(s["lat"]), "plain_latency": pct(p["lat"]),
        "plain_graphs_per_s": plain_gps, "speedup_vs_plain": served_gps / plain_gps,
        "served_points_iter_per_s": ranks.sum(s["samples"] * sb.iters / s["span"]),
        "server": {k: stats[k] for k in ("peak_active", "peak_device_bytes", "budget_waits", "evictions", "steps",
                                         "launch_s", "upload_s", "wait_s", "retire_s", "idle_s", "contexts_created",
                                         "create_s")},
        "submit_seconds": s["submit_s"], "arrivals_late": s["late"],
        "bit_exact_vs_plain": s["exact"],
        "clocks": clock_info,
        "capacity_and_latency": served_measure(args, ranks),
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.quick:
        args.e2e_jobs, args.no_batched, args.no_served, args.no_cpu_baseline = 0, True, True, True
    ranks = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, ranks)
        elif args.workload == "batched":
            run_batched(args, ranks)
        elif args.workload == "served":
            run_served(args, ranks)
        elif args.workload == "render":
            run_render(args, ranks)
        elif args.workload == "advect":
            run_advect(args, ranks)
        else:
            run_ours(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
