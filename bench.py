"""Benchmark: spectral paths/s of the CUDA Path-Traced sample loop on B200.

One "step" is one pass of the hot path over one batch of synthetic input:

* ``--workload batch`` (default): 64 seeded random stones x 9 tilts at 128x128 with spp
  drawn from {32, 64, 128, 256} -- one persistent launch per step (about 1.1e9 paths);
* ``--workload frame``: the 256x256, 64 spp round-brilliant frame (4,194,304 paths;
  Diamond, D65 hemisphere with a 20-degree head shadow, depth 32);
* ``--workload stress``: the anisotropic stress frame, 512x512 x 256 spp (67,108,864
  paths) of a uniaxial pleochroic emerald-cut stone with its optic axis tilted 30
  degrees, depth 64.
* ``--workload sun``: the extended transport on a 256x256, 64 spp round brilliant with its
  table and girdle frosted and a dimple ground into the table, under the DaylightSun
  model (frosted next-event estimation toward the sun's disc), depth 32.
* ``--workload display``: the display step after the path on a 1920x1080 frame of 16 spp
  XYZ sums (the reference's denoise bench: round brilliant at (0.60, 0.45, 2.4, 42 deg),
  path signature at n_d 1.76, seeded noise in [0, 2) per channel): average, 5 A-Trous
  passes with the sRGB tone-map fused into the last, guides cached per pose.  The metric
  is display frames/s; under torchrun every rank displays its own frame (replicas).

Under torchrun (N > 1) every rank traces its own disjoint absolute sample range of the
same workload (weak scaling), and the per-pixel f64 sums are gathered to rank 0 over
NCCL and folded in ascending first-sample order (the deterministic merge of the
reference's indicatrix-dispatch).

Printed on rank 0: one JSON line with the contract's keys, plus ``roofline`` (FP32 FMA
pipe, measured by a probe kernel) and ``cpu_baseline`` (the CPU oracle on the host
cores).  ``--impl reference`` times the reference's CPU implementation of the path (the
oracle restatement, all host threads) on the same workload instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "spectral paths/s"
UNIT = "paths/s"
L2_FLUSH_BYTES = 512 << 20  # > the 126 MB L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch", choices=["frame", "batch", "stress", "sun", "display", "surrogate"])
    ap.add_argument("--precision", default="fast", choices=["fast", "exact"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--stones", type=int, default=64,
                    help="batch workload: the first N of the 64 seeded stones (profiling small case)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="pin the kernel variant (budget + 3 * shape): the batch plan's instead of "
                         "autotuning, the frame's instead of the backend's default")
    ap.add_argument("--designs", type=int, default=16384, help="surrogate workload: training designs")
    ap.add_argument("--population", type=int, default=4096, help="surrogate workload: candidates per generation")
    ap.add_argument("--generations", type=int, default=50, help="surrogate workload: search generations")
    ap.add_argument("--epochs", type=int, default=300, help="surrogate workload: training epochs per member")
    ap.add_argument("--members", type=int, default=4, help="surrogate workload: ensemble members")
    ap.add_argument("--gemm-only", action="store_true",
                    help="surrogate workload: time the fused linear layer's GEMM shapes only (profiling case)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------
# Workloads
# ----------------------------------------------------------------------------------
def frame_workload(builder=None):
    from indicatrix_b200 import workloads

    fs = workloads.round_brilliant_frame(256, 256, 32, builder=builder)
    return [(fs, 64)], {"workload": "round brilliant frame 256x256 x 64 spp", "pixels": 65536,
                        "spp": 64, "planes": int(fs.planes.shape[0]), "material": "diamond",
                        "environment": "D65 hemisphere, 20 deg head shadow", "max_depth": 32}


def stress_workload(builder=None):
    from indicatrix_b200 import workloads

    fs = workloads.anisotropic_stress_frame(512, 512, 64, builder=builder)
    return [(fs, 256)], {"workload": "anisotropic stress frame 512x512 x 256 spp", "pixels": 512 * 512,
                         "spp": 256, "planes": int(fs.planes.shape[0]),
                         "material": "uniaxial corundum (n_o 1.768, n_e 1.760, Sellmeier o/e), optic axis "
                                     "tilted 30 deg, o/e spline absorption 0-8 /cm",
                         "stone": "emerald step cut, 3+3 tiers, 49 facets",
                         "environment": "D65 hemisphere, 20 deg head shadow", "max_depth": 64}


def sun_workload(builder=None):
    from indicatrix_b200 import workloads

    fs = workloads.carved_sun_frame(256, 256, 32, builder=builder)
    return [(fs, 64)], {"workload": "carved frosted round brilliant under the sun 256x256 x 64 spp",
                        "pixels": 65536, "spp": 64, "planes": int(fs.planes.shape[0]), "material": "diamond",
                        "stone": "table and girdle frosted, a 0.11 ball dimple in the table",
                        "environment": "DaylightSun, light yaw 0.4 pitch 0.5, frosted next-event estimation",
                        "max_depth": 32}


def batch_workload(n_stones: int = 64, builder=None):
    from indicatrix_b200 import workloads

    # The first n_stones of the same seeded sequence (64 is the benchmark; fewer make the
    # small case a profiler captures).
    stones = workloads.random_stones(64)[:n_stones]
    items = []
    for st in stones:
        for tilt in workloads.TILTS_DEG:
            items.append((workloads.tilted_scene(st, tilt, 128, 128, 32, builder=builder), st.spp))
    paths = sum(fs.width * fs.height * spp for fs, spp in items)
    return items, {"workload": f"{n_stones} random stones x 9 tilts x 128x128, spp in {{32,64,128,256}}",
                   "stones": n_stones, "tilts": 9, "paths": paths, "max_depth": 32}


def workload_items(args, builder=None):
    if args.workload == "batch":
        return batch_workload(args.stones, builder)
    return {"frame": frame_workload, "stress": stress_workload, "sun": sun_workload}[args.workload](builder)


# ----------------------------------------------------------------------------------
# CPU baseline: the oracle on the host cores, on a bounded sample of the workload.
# ----------------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ix_oracle

    ix_oracle.build()
    return ix_oracle


def cpu_entries(items, per_item: int, seed: int):
    """A seeded sample with the GPU step's path distribution: `per_item` pixels drawn
    uniformly from every scene of the workload, each with all its samples (so every scene
    contributes in proportion to its paths)."""
    rng = np.random.default_rng(seed)
    rows = []
    for k, (fs, spp) in enumerate(items):
        for p in rng.integers(0, fs.width * fs.height, per_item):
            rows.append((k, int(p), spp))
    return np.array(rows, np.uint32)


def cpu_trace(ixo, scenes, entries, threads):
    lib = ixo.simd_lib()
    t0 = time.perf_counter()
    paths, _, _ = ixo.trace_pixel_set(scenes, entries, 0, threads, lib)
    return paths, time.perf_counter() - t0


def cpu_plan(ixo, items, scenes, seconds: float, threads: int, seed: int):
    """Pixels per scene sized from a short calibration run so that tracing the sample on
    `threads` host threads takes about `seconds`."""
    probe = cpu_entries(items, max(2, 1024 // len(items)), seed ^ 0x5A5A)
    paths, dt = cpu_trace(ixo, scenes, probe, threads)
    rate = paths / max(dt, 1e-3)
    mean_spp = sum(spp for _, spp in items) / len(items)
    return max(1, int(round(rate * seconds / (mean_spp * len(items)))))


def cpu_kind(ixo):
    if ixo.simd_lib().ixo_simd_build():
        return ("the oracle (the reference CPU tracer restated in C++, -O3, with its AVX2 slab-scan and "
                "8-lane exp twins)")
    return "the oracle (the reference CPU tracer restated in C++, -O3, scalar)"


def cpu_baseline(items, seconds: float):
    """All-core and single-core rates of the oracle on the workload's path distribution."""
    ixo = _oracle()
    threads = os.cpu_count() or 1
    scenes = [fs.to_abi() for fs, _ in items]
    per_item = cpu_plan(ixo, items, scenes, seconds, threads, seed=101)
    entries = cpu_entries(items, per_item, 101)
    paths, dt = cpu_trace(ixo, scenes, entries, threads)
    per_item1 = cpu_plan(ixo, items, scenes, max(2.0, seconds / 3.0), 1, seed=202)
    one = cpu_entries(items, per_item1, 202)
    p1, d1 = cpu_trace(ixo, scenes, one, 1)
    return {"value": paths / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "single_core": p1 / d1,
            "sample": f"{per_item} pixels drawn uniformly from each of the {len(items)} scenes of the workload, "
                      f"all their samples ({paths} paths, {dt:.1f} s on {threads} host threads; single core: "
                      f"{per_item1} pixels per scene, {p1} paths, {d1:.1f} s); {cpu_kind(ixo)}"}


def loaded_native_libraries():
    """Shared objects under this repository mapped into this process (relative paths)."""
    names = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if line.strip() else ""
                if path.startswith(ROOT) and path.endswith(".so"):
                    names.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(names)


def count_flops(items):
    ixo = _oracle()
    total_f, total_p = 0, 0
    div = sqrt = transc = 0
    step = max(1, len(items) // 8)
    for fs, spp in items[::step]:
        sc = fs.to_abi()
        n_pix = fs.width * fs.height
        # A pixel stride coprime with the width, so the sample spreads over every column.
        stride = max(1, n_pix // (8192 // max(1, spp // 16)))
        while math.gcd(stride, fs.width) != 1:
            stride += 1
        c = ixo.count_flops(sc, 0, n_pix, stride, 0, spp)
        total_f += c.flops()
        total_p += c.paths
        div, sqrt, transc = div + c.div, sqrt + c.sqrt, transc + c.transcendental
    return total_f / total_p, {"sample_paths": total_p, "div_per_path": div / total_p,
                               "sqrt_per_path": sqrt / total_p, "transcendental_per_path": transc / total_p}


# ----------------------------------------------------------------------------------
# Reference arm
# ----------------------------------------------------------------------------------
REFERENCE_RUN_SECONDS = 150.0  # the whole --steps K --warmup W run of the reference arm


def run_reference(args, items, cfg):
    """The reference's CPU implementation of the path (restated in C++, see cpu_kind) on
    every host thread: each step traces a fresh seeded sample with the GPU step's path
    distribution, sized so the whole run takes about REFERENCE_RUN_SECONDS.  Scenes are
    built by the oracle's own host formulas: nothing of the CUDA library is loaded."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    ixo = _oracle()
    threads = os.cpu_count() or 1
    scenes = [fs.to_abi() for fs, _ in items]
    per_step = REFERENCE_RUN_SECONDS / max(1, args.steps + args.warmup)
    per_item = cpu_plan(ixo, items, scenes, per_step, threads, seed=7)
    for w in range(args.warmup):
        cpu_trace(ixo, scenes, cpu_entries(items, per_item, 1000 + w), threads)
    times, paths = [], 0
    for k in range(args.steps):
        p, dt = cpu_trace(ixo, scenes, cpu_entries(items, per_item, 2000 + k), threads)
        times.append(dt)
        paths += p
    value = paths / sum(times)
    libs = loaded_native_libraries()
    if any("libix_cuda" in n for n in libs):
        raise RuntimeError(f"the reference arm loaded the CUDA library: {libs}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"per step {per_item} fresh pixels drawn uniformly from each of the "
                                   f"{len(items)} scenes of the workload, all their samples ({paths} paths in "
                                   f"{args.steps} steps); {cpu_kind(ixo)}; the reference (Rust) cannot be "
                                   "built here"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_libraries": libs,
    }), flush=True)


# ----------------------------------------------------------------------------------
# The display step after the path (guide pass, A-Trous denoise, tone-map)
# ----------------------------------------------------------------------------------
DISPLAY_METRIC, DISPLAY_UNIT = "display frames/s", "frames/s"
HBM_PEAK_FALLBACK_GBS = 6650.0


def display_workload():
    from indicatrix_b200 import materials, workloads
    from indicatrix_b200.backend import FrameScene, camera_new

    w, h, spp = 1920, 1080, 16
    base = workloads.round_brilliant_frame(8, 8)
    # n_d exactly 1.76 (the reference bench's signature index): a flat Cauchy index.
    mat = materials.isotropic(materials.cauchy(1.76, 0.0, 0.0))
    fs = FrameScene(camera_new(0.60, 0.45, 2.4, 42.0), w, h, base.planes, mat, 32, base.environment)
    rng = np.random.default_rng(0x9E3779B9)
    # Per channel a value in [0, 2) on the reference bench's 1/32768 grid, summed over spp.
    color = (rng.integers(0, 65536, size=(h, w, 3), dtype=np.uint32).astype(np.float32) / np.float32(32768.0))
    accum = (color * np.float32(spp)).astype(np.float32)
    cfg = {"workload": "display step 1920x1080 from 16 spp XYZ sums: average, 5 A-Trous passes with path "
                       "signature, sRGB tone-map", "width": w, "height": h, "spp": spp, "passes": 5,
           "signature_n_d": 1.76, "stone": "standard round brilliant, 74 facets",
           "pose": "yaw 0.60, pitch 0.45, distance 2.4, fov 42 deg"}
    return fs, accum, spp, cfg


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured"
    return HBM_PEAK_FALLBACK_GBS, "fallback"


def display_cpu(fs, accum, spp, frames: int):
    """The oracle's display step (guides at n_d 1.76, denoise, tone-map) on all host
    threads: seconds per frame, the guides timed once outside."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ix_oracle

    ix_oracle.build()
    threads = os.cpu_count() or 1
    d, n, f, s = ix_oracle.generate_guide_buffers(fs.width, fs.height, fs.camera, fs.planes, 1.76, threads)
    times = []
    for _ in range(frames):
        t0 = time.perf_counter()
        ix_oracle.denoise_and_tonemap_frame(accum, spp, d, n, f, s, threads=threads)
        times.append(time.perf_counter() - t0)
    return sum(times) / len(times), threads


def display_flops_per_pixel_pass(fs, accum, spp):
    """Algorithmic FP32 operations per pixel-pass of the A-Trous denoise, counted by the
    oracle's counting build on a 480x270 crop around the stone of the same frame."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ix_oracle

    ix_oracle.build()
    cw, ch = 480, 270
    x0, y0 = (fs.width - cw) // 2, (fs.height - ch) // 2
    d, n, f, s = ix_oracle.generate_guide_buffers(fs.width, fs.height, fs.camera, fs.planes, 1.76)
    crop = (slice(y0, y0 + ch), slice(x0, x0 + cw))
    avg = (accum[crop] * (np.float32(1.0) / np.float32(spp))).astype(np.float32)
    c = ix_oracle.count_denoise_flops(avg, d[crop], n[crop], f[crop], s[crop], spp)
    return c.flops() / c.paths, float(np.mean(f[crop] >= 0))


def run_display_reference(args, fs, accum, spp, cfg):
    rank, _, _ = dist_env()
    if rank != 0:
        return
    for _ in range(max(0, min(args.warmup, 1))):
        display_cpu(fs, accum, spp, 1)
    sec, threads = display_cpu(fs, accum, spp, args.steps)
    value = 1.0 / sec
    print(json.dumps({
        "impl": "reference", "metric": DISPLAY_METRIC, "value": value, "unit": DISPLAY_UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": DISPLAY_UNIT, "cores": threads, "kind": "port",
                         "sample": f"the whole 1920x1080 frame per step ({args.steps} frames): the reference's "
                                   "denoise and tone-map (Rust, not buildable here) restated in C++, all host "
                                   "threads"},
        "e2e": {"value": value, "unit": DISPLAY_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main_display(args):
    rank, world, local = dist_env()
    fs, accum, spp, cfg = display_workload()
    cfg["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
    if args.impl == "reference":
        run_display_reference(args, fs, accum, spp, cfg)
        return
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from indicatrix_b200 import abi, display
    from indicatrix_b200.backend import GpuBackend

    precision = abi.PRECISION_EXACT if args.precision == "exact" else abi.PRECISION_FAST
    backend = GpuBackend.acquire(device=local, precision=precision)
    if not backend.available:
        raise RuntimeError("libix_cuda.so could not create a backend")
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    d_acc = torch.from_numpy(accum).to(dev)
    d_rgba = torch.empty((fs.height, fs.width, 4), dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sc = fs.to_abi()

    def step():
        if not display.display_frame_device(backend, sc, spp, d_acc.data_ptr(), d_rgba.data_ptr(), True,
                                            stream_ptr=stream.cuda_stream):
            raise RuntimeError(f"display declined: {backend.last_lost_reason()}")

    for _ in range(args.warmup):  # the first call computes and caches the guides
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    atrous_ms, launches = [], 0
    for k in range(args.steps):
        flush.zero_()  # the ~120 MB working set fits L2: flush between timed steps
        starts[k].record(stream)
        step()
        ends[k].record(stream)
        t = display.last_timing(backend)  # the A-Trous kernels' events on the same stream
        atrous_ms.append(t.atrous_ms)
        launches += t.launches
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    mean_ms = sum(step_ms) / len(step_ms)
    if world > 1:
        t = torch.tensor([mean_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        mean_ms = float(t.item())
    value = world / (mean_ms * 1e-3)

    # End to end through the public host API: H2D of the f32 sums, D2H of the RGBA8.
    e2e_ms = []
    host_rgba = np.zeros((fs.height, fs.width, 4), np.uint8)  # the caller's frame buffer, reused
    for k in range(max(1, args.warmup // 2) + min(args.steps, 50)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = display.display_frame(backend, fs, spp, accum, True, out=host_rgba)
        if out is None:
            raise RuntimeError(f"display declined: {backend.last_lost_reason()}")
        if k >= max(1, args.warmup // 2):
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_mean = sum(e2e_ms) / len(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_mean], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_mean = float(t.item())
        torch.distributed.destroy_process_group()
    pixels = fs.width * fs.height

    if rank == 0:
        passes = 5
        # Algorithmic bytes of one A-Trous launch: per pixel the centre's colour (16 B),
        # packed guides (16 + 8 B) and the colour written (16 B); the last pass writes
        # RGBA8 (4 B) instead.  Averaged over the 5 launches of a frame.
        bytes_per_launch = pixels * (4 * 56 + 44) / passes
        atrous_launch_ms = statistics.mean(atrous_ms) / passes
        achieved = bytes_per_launch / (atrous_launch_ms * 1e-3) / 1e9
        peak, peak_kind = hbm_peak()
        flops_pp, fg = display_flops_per_pixel_pass(fs, accum, spp)
        line = {
            "metric": DISPLAY_METRIC, "value": value, "unit": DISPLAY_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**cfg, "precision": args.precision,
                       "l2": "512 MB buffer written between timed steps (outside the step events)",
                       "megapixels_per_s": value * pixels / 1e6},
            "e2e": {"value": world / (e2e_mean * 1e-3), "unit": DISPLAY_UNIT,
                    "h2d_bytes_per_step": pixels * 12, "d2h_bytes_per_step": pixels * 4, "ms_per_step": e2e_mean},
            "gpu_launches": launches,
            # traffic: DRAM read + write bytes of one A-Trous launch (passes 1-4) from the
            # ncu capture of this workload at full size (profiles/atrous_display_1080p.md).
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": 56.3e6,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "kernel": "atrous_pass_kernel", "launch_ms": atrous_launch_ms,
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "flops_per_pixel_pass": flops_pp, "foreground_fraction": fg},
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            sec, threads = display_cpu(fs, accum, spp, 1)
            line["cpu_baseline"] = {"value": 1.0 / sec, "unit": DISPLAY_UNIT, "cores": threads, "kind": "port",
                                    "sample": "one whole 1920x1080 frame: the C++ oracle's denoise + tone-map on "
                                              f"{threads} host threads ({sec:.2f} s)"}
        print(json.dumps(line), flush=True)
    backend.close()


# ----------------------------------------------------------------------------------
# Surrogate-screened design search (--workload surrogate)
# ----------------------------------------------------------------------------------
SURROGATE_METRIC = "design evaluations/s"
SURROGATE_UNIT = "designs/s"


def tensor_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            v = json.load(f).get("bf16_tflops")
        if v:
            return float(v), "measured"
    return 1590.0, "fallback"


def time_gemm(torch, m, n, k, reps=50):
    """CUDA-event time of one fused linear layer (tcgen05 GEMM + bias + SiLU epilogue) of
    shape m x n x k on the current stream, after 3 warm-up launches: ms per launch."""
    from indicatrix_b200 import surrogate as S

    lib, st = S._lib(), torch.cuda.current_stream().cuda_stream
    x = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    w = (torch.randn(n, k, device="cuda") / math.sqrt(k)).to(torch.bfloat16)
    b = torch.zeros(n, device="cuda")
    hb = torch.empty(m, n, dtype=torch.bfloat16, device="cuda")
    z = torch.empty(m, n, device="cuda")

    def launch():
        if lib.ix_mlp_linear(m, n, k, x.data_ptr(), k, w.data_ptr(), b.data_ptr(), 1, z.data_ptr(), None,
                             hb.data_ptr(), st) != 0:
            raise RuntimeError("GEMM launch failed")

    for _ in range(3):
        launch()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        launch()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main_surrogate(args):
    """Config 5 at reduced scale: an evolutionary design search whose candidates the
    trained ensemble scores (the tracer scoring the ones it disagrees on and re-rendering
    the best 64 of each generation), against the same search scored by the tracer alone;
    both timed end to end (host designs in, host metrics out, device work synchronised)."""
    rank, world, local = dist_env()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned surrogate: its "
                              "cut optimiser scores candidates with the analytic metrics"}), flush=True)
        return
    if rank != 0:
        return  # replicas only: the search runs on one GPU
    import torch

    torch.cuda.set_device(local)
    from indicatrix_b200 import surrogate as S
    from indicatrix_b200.backend import GpuBackend

    if args.gemm_only:
        peak, peak_kind = tensor_peak()
        rows = []
        for m, n, k in [(4096, 256, 256), (65536, 256, 256), (4096, 27, 256), (4096, 256, 12)]:
            ms = time_gemm(torch, m, n, k, reps=max(1, args.steps))
            tf = 2 * m * n * k / (ms * 1e-3) / 1e12
            rows.append({"shape": [m, n, k], "launch_ms": ms, "tflops": tf, "frac": tf / peak})
        print(json.dumps({"workload": "surrogate GEMM layers (fused bias + SiLU epilogue)", "peak": peak,
                          "peak_source": f"{peak_kind} cuBLAS bf16 burst", "layers": rows}), flush=True)
        return

    backend = GpuBackend.acquire(device=local)
    if not backend.available:
        raise RuntimeError("libix_cuda.so could not create a backend")
    spec = S.RenderSpec(width=32, height=32, spp=64)
    final_spec = S.RenderSpec(width=32, height=32, spp=1024, sample_offset=1 << 21)
    t0 = time.perf_counter()
    train = S.sample_designs(args.designs, 2)
    y = S.evaluate_designs(backend, train, spec)
    data_s = time.perf_counter() - t0
    hold = S.sample_designs(512, 3)
    y_hold = S.evaluate_designs(backend, hold, S.RenderSpec(width=32, height=32, spp=1024, sample_offset=1 << 20))
    scales = S.tilt_means(y).mean(axis=0)
    ens = S.SurrogateEnsemble(args.members, seed=0)
    t0 = time.perf_counter()
    losses = ens.fit(S.normalize(train), y, epochs=args.epochs, batch=4096, lr=1e-3)
    fit_s = time.perf_counter() - t0
    pm, s_hold, dis = ens.score(S.normalize(hold), scales)
    th, tp = S.tilt_means(y_hold), S.tilt_means(pm)
    s_true = S.score(y_hold, scales)
    pred_rel = np.abs(tp - th) / th
    cfg = S.SearchConfig(population=args.population, generations=args.generations)
    warm = S.SearchConfig(population=args.population, generations=3, seed=99)
    S.screened_search(backend, ens, scales, warm, spec)
    S.traced_search(backend, scales, warm, spec)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = S.launches
    r1 = S.screened_search(backend, ens, scales, cfg, spec)
    screened_launches = S.launches - l0
    r2 = S.traced_search(backend, scales, cfg, spec)
    clk = clocks.stop()
    fin = S.evaluate_designs(backend, np.stack([r1.best_design, r2.best_design]), final_spec)
    fs = S.score(fin, scales)
    pred_final = ens.predict(S.normalize(r1.best_design[None]))[0]
    # The GEMM's roofline: the training step's 4096 x 256 x 256 layer and a large layer.
    g_small = time_gemm(torch, 4096, 256, 256)
    g_large = time_gemm(torch, 65536, 256, 256, reps=20)
    peak, peak_kind = tensor_peak()
    ach_small = 2 * 4096 * 256 * 256 / (g_small * 1e-3) / 1e12
    ach_large = 2 * 65536 * 256 * 256 / (g_large * 1e-3) / 1e12
    gens = args.generations
    bytes_in = args.population * 12 * 4  # designs uploaded per generation (bf16 path: f32 first)
    bytes_out = args.members * args.population * 27 * 4 + (r1.traced // max(1, gens)) * 27 * 4
    line = {
        "metric": SURROGATE_METRIC, "value": r1.evals_per_s, "unit": SURROGATE_UNIT, "n_gpus": 1,
        "steps": gens, "warmup": 3, "ms_per_step": r1.seconds / gens * 1e3, "higher_is_better": True,
        "scaling": "replicas only", "vs_baseline": None, "dtype": "bf16 (MLP, FP32 accumulation); f32 (tracer)",
        "data": "synthetic: seeded designs uniform over the 12-parameter box, metrics traced by this library",
        "config": {"workload": "surrogate-screened evolutionary design search (config 5, reduced scale)",
                   "population": args.population, "generations": gens, "retraced_per_generation": 64,
                   "fallback_disagreement": 0.02, "ensemble_members": args.members,
                   "network": "12-256-256-256-27 SiLU, BF16 weights/activations, FP32 accumulation",
                   "search_render": "32x32, 64 spp, 9 tilts 0-40 deg (split-half image metrics)",
                   "training_set": f"{args.designs} designs at 32x32, 64 spp, 9 tilts; Adam lr 1e-3 -> 5e-5, "
                                   f"batch 4096, {args.epochs} epochs per member",
                   "final_render": "32x32, 1024 spp, 9 tilts, a disjoint sample range",
                   "scale_note": "config 4/5 name 200k designs at 64x64 64 spp and re-renders at 256x256 "
                                 "1024 spp; this run keeps the network, population, generations, top-64 "
                                 "re-trace and fallback rule and reduces the render sizes and the dataset",
                   "l2": "not flushed: a generation's working set is host-driven and re-uploaded"},
        "e2e": {"value": r1.evals_per_s, "unit": SURROGATE_UNIT, "h2d_bytes_per_step": bytes_in,
                "d2h_bytes_per_step": bytes_out,
                "note": "the search is host-driven: value and e2e are the same wall-clock measurement"},
        "plain_tracer_evals_per_s": r2.evals_per_s,
        "speedup_vs_plain_tracing": r1.evals_per_s / r2.evals_per_s,
        "final": {"screened_score_1024spp": float(fs[0]), "traced_only_score_1024spp": float(fs[1]),
                  "screened_over_traced_only": float(fs[0] / fs[1]),
                  "screened_search_metrics_vs_1024spp_rel_err": S.relative_error(r1.best_metrics, fin[0]).tolist(),
                  "surrogate_prediction_vs_1024spp_rel_err": S.relative_error(pred_final, fin[0]).tolist(),
                  "traced_only_search_metrics_vs_1024spp_rel_err": S.relative_error(r2.best_metrics, fin[1]).tolist()},
        "search": {"screened_seconds": r1.seconds, "traced_only_seconds": r2.seconds, "traced": r1.traced,
                   "fallbacks": r1.fallbacks, "fallback_fraction": r1.fallbacks / r1.evaluations,
                   "screened_history": r1.history, "traced_only_history": r2.history},
        "holdout": {"designs": 512, "render": "32x32, 1024 spp",
                    "prediction_rel_err_median": np.median(pred_rel, axis=0).tolist(),
                    "prediction_rel_err_p90": np.percentile(pred_rel, 90, axis=0).tolist(),
                    "score_rel_err_median": float(np.median(np.abs(s_hold - s_true) / s_true)),
                    "disagreement_median": float(np.median(dis)),
                    "fraction_over_fallback": float(np.mean(dis > 0.02))},
        "training": {"dataset_seconds": data_s,
                     "dataset_paths_per_s": args.designs * spec.paths_per_design() / data_s,
                     "fit_seconds": fit_s, "loss_first": [l[0] for l in losses],
                     "loss_last": [l[-1] for l in losses]},
        "gpu_launches": screened_launches,
        "roofline": {"bound": "tensor", "achieved": ach_small, "peak": peak, "unit": "TFLOP/s",
                     "frac": ach_small / peak, "traffic": None, "peak_source": f"{peak_kind} cuBLAS bf16 burst",
                     "kernel": "umma_gemm_kernel (fused linear layer)", "shape": [4096, 256, 256],
                     "launch_ms": g_small, "large_layer": {"shape": [65536, 256, 256], "launch_ms": g_large,
                                                           "achieved": ach_large, "frac": ach_large / peak}},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    backend.close()


# ----------------------------------------------------------------------------------
# Our arm
# ----------------------------------------------------------------------------------
# DRAM read + write bytes per pixel of one trace-kernel launch, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on a small case of the same kernel, and
# how that case was taken.
DRAM_BYTES_PER_PIXEL = {"batch": 124.6, "stress": 19.7}
TRAFFIC_SOURCE = {
    "batch": "ncu --set full capture of the task-loop batch kernel (32-warp budget) on the first 4 stones x "
             "9 tilts (589,824 pixels), per-pixel bytes scaled to this launch's pixels",
    "stress": "ncu capture of the stress frame kernel at 128x128 x 256 spp, per-pixel bytes scaled to "
              "this launch's pixels",
}


def device_tensor(torch, ptr: int, n: int, dev):
    """A zero-copy torch view of `n` f64 at device address `ptr` (the library's buffer)."""

    class _Buf:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                    "strides": None}

    return torch.as_tensor(_Buf(), device=dev)

def main():
    args = parse()
    if args.workload == "display":
        main_display(args)
        return
    if args.workload == "surrogate":
        main_surrogate(args)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        # Scenes from the oracle's host formulas (Camera::new, the lighting presets): the
        # reference arm runs the reference's CPU path only.
        items, cfg = workload_items(args, builder=_oracle())
        cfg["parallelism"] = f"sample-range shards x{world}" if world > 1 else "single GPU"
        run_reference(args, items, cfg)
        return
    items, cfg = workload_items(args)
    cfg["parallelism"] = f"sample-range shards x{world}" if world > 1 else "single GPU"

    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from indicatrix_b200 import abi
    from indicatrix_b200.backend import GpuBackend

    precision = abi.PRECISION_EXACT if args.precision == "exact" else abi.PRECISION_FAST
    # Frames: a pinned kernel variant goes to the backend (0 = its default per scene);
    # the batch plan pins or autotunes its own below.
    frame_variant = args.variant + 1 if (args.variant >= 0 and args.workload != "batch") else 0
    backend = GpuBackend.acquire(device=local, precision=precision, kernel_variant=frame_variant)
    if not backend.available:
        raise RuntimeError("libix_cuda.so could not create a backend")

    # Device-resident inputs and outputs.
    total_paths = sum(fs.width * fs.height * spp for fs, spp in items)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    # A dedicated (non-default) stream: the library enqueues on exactly this stream and
    # the step events are recorded on it.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    # Disjoint absolute sample ranges per rank: rank r traces [r spp, (r + 1) spp) of every
    # scene, so rank order is first-sample order for the fold.
    dev_items = []
    plan = None
    if args.workload == "batch":
        from indicatrix_b200.backend import BatchPlan

        plan = BatchPlan(backend, [(fs, rank * spp, spp) for fs, spp in items])
        if args.variant >= 0:
            if not plan.set_variant(args.variant):
                raise RuntimeError(f"kernel variant {args.variant} is not available in this build")
            cfg["pinned_variant"] = args.variant
        else:
            cfg["autotuned_variant"] = plan.autotune(reps=1)
        n_out = sum(fs.width * fs.height * 3 for fs, _ in items)
        result = device_tensor(torch, plan.device_output(), n_out, dev)
    else:
        from indicatrix_b200 import abi

        for fs, spp in items:
            sc = fs.to_abi()
            # Every array of the scene goes to the device: the device entry reads no host memory.
            planes = torch.from_numpy(np.ascontiguousarray(fs.planes, np.float32)).to(dev)
            sc.planes = C.cast(C.c_void_p(planes.data_ptr()), C.POINTER(C.c_float))
            keep = [planes]
            if fs.facet_finishes is not None:
                fin = torch.from_numpy(np.ascontiguousarray(fs.facet_finishes, np.uint8)).to(dev)
                sc.facet_finishes = C.cast(C.c_void_p(fin.data_ptr()), C.POINTER(C.c_uint8))
                keep.append(fin)
            if fs.tools:
                raw = np.frombuffer(bytes((abi.Tool * len(fs.tools))(*fs.tools)), np.uint8).copy()
                tools = torch.from_numpy(raw).to(dev)
                sc.tools = C.cast(C.c_void_p(tools.data_ptr()), C.POINTER(abi.Tool))
                keep.append(tools)
            out = torch.zeros(fs.width * fs.height * 3, dtype=torch.float64, device=dev)
            dev_items.append((sc, keep, out, spp, fs))
        result = dev_items[0][2]

    def step(k):
        if plan is not None:
            plan.run(stream.cuda_stream)
        for sc, _planes, out, spp, _fs in dev_items:
            rc = backend.accumulate_device(sc, rank * spp, spp, out.data_ptr(), False, stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(f"device trace declined: {backend.last_lost_reason()}")
        if world > 1:
            # The exchange step: every rank's per-pixel f64 sums to rank 0 (NCCL gather),
            # folded there in first-sample order.
            from indicatrix_b200.dispatch import gather_fold

            gather_fold(result)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()  # L2 flush between timed iterations (outside the step events)
        starts[k].record(stream)
        step(k)
        ends[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    mean_ms = sum(step_ms) / len(step_ms)
    if world > 1:
        t = torch.tensor([mean_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        mean_ms = float(t.item())
    value = world * total_paths / (mean_ms * 1e-3)
    # Kernels of this library per step: the trace launch(es), plus the rounding of the
    # fixed-point sums after each path-pool launch.
    if plan is not None:
        launches_per_step = 2 if plan.variant >= 3 else 1
    else:
        launches_per_step = backend.last_timing().launches

    # End-to-end through the public API with host buffers (H2D scenes and planes, D2H
    # per-pixel sums): try_accumulate for the frame, try_accumulate_batch for the batch.
    from indicatrix_b200.backend import GpuBatchItem

    e2e_ms = []
    accs = [np.zeros((fs.height, fs.width, 3), np.float64) for fs, _ in items]
    for k in range(max(1, args.warmup // 2) + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if plan is not None:
            batch = [GpuBatchItem(fs, rank * spp, spp, acc) for (fs, spp), acc in zip(items, accs)]
            if backend.try_accumulate_batch_cancellable(batch) != 0:
                raise RuntimeError(f"e2e batch declined: {backend.last_lost_reason()}")
        else:
            for (fs, spp), acc in zip(items, accs):
                if not backend.try_accumulate(fs, rank * spp, spp, acc):
                    raise RuntimeError(f"e2e trace declined: {backend.last_lost_reason()}")
        t1 = time.perf_counter()
        if k >= max(1, args.warmup // 2):
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_mean = sum(e2e_ms) / len(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_mean], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_mean = float(t.item())
    h2d = sum(int(fs.planes.shape[0]) * 16 for fs, _ in items)
    d2h = sum(fs.width * fs.height * 3 * 8 + 8 for fs, _ in items)

    if rank == 0:
        peak = backend.probe_fp32_peak()
        flops_per_path, flop_info = count_flops(items)
        # dominant kernel: the trace megakernel; per-launch algorithmic FLOPs / duration
        achieved = flops_per_path * total_paths / (mean_ms * 1e-3)
        # DRAM bytes (read + write) per pixel of the trace kernel, from one ncu capture of a
        # small case of the same kernel and variant, scaled to this launch by its pixels
        # (the per-pixel sums are the only DRAM traffic; planes and paths stay on chip).
        dram_bytes_per_pixel = DRAM_BYTES_PER_PIXEL.get(args.workload)
        total_pixels = sum(fs.width * fs.height for fs, _ in items)
        traffic = dram_bytes_per_pixel * total_pixels if dram_bytes_per_pixel is not None else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**cfg, "precision": args.precision,
                       "l2": "512 MB buffer written between timed steps (outside the step events)",
                       "spectral_samples_per_s": 8.0 * value},
            "e2e": {"value": world * total_paths / (e2e_mean * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_mean},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                         "traffic": traffic,
                         "traffic_source": TRAFFIC_SOURCE.get(args.workload),
                         "peak_source": "measured by the FP32 FMA-chain probe kernel (FMA = 2 FLOP) "
                                        "in this run; MEASURED_PEAKS.json has no non-tensor FP32 figure",
                         "flops_per_path": flops_per_path, "flop_count": flop_info},
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(items, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    backend.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
