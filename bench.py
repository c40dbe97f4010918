#!/usr/bin/env python3
"""Benchmark of the scene-flush / trace hot path on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload trace|build|batch|flush]

Workloads (seeded synthetic inputs with the shapes of the benchmark configurations; no dataset):
  trace   (default, the headline) the plain brick-DDA trace: a 128^3-voxel world of 16^3 bricks,
          30 % of the bricks occupied by thresholded value noise, voxel materials uniform in
          [1, 64], 1 % of the occupied bricks emissive (power log-normal(0, 1)), brick keys in the
          device hash table at load factor 0.5; 512 x 512 pinhole camera, 1 spp, 4 bounces,
          light-tree NEE with MIS; fp32 radiance. A step is one render call; value = Mrays/s with
          the rays counted on the device (primary + bounce + shadow).
  build   the light-tree build over 4,194,304 brick light records (brick coords uniform in a
          1024^3-brick grid, 16^3-brick render groups, power log-normal(0, 1) split over the faces);
          value = Mleaves/s.
  batch   64 scenes (brick counts log-uniform in [1k, 500k], square viewports 256/512/1024, 2 spp,
          4 bounces): every scene's light-tree rebuild + the trace of every view as one CUDA graph
          launch, against the same work one scene at a time through the plain C ABI.
  flush   the scene flush of the 2M-brick world: the incremental flush after re-uploading 1 % of
          the bricks (value, ms), the first flush, a full rebuild and a light-tree-only flush.
The trace line carries the other measurements as objects: `build` (the 4M-record build with its
roofline and stage times, and the 4,096-record plain build in ms), `large` (the 2M-brick world at
1920 x 1080, 4 spp, 6 bounces: flush and frame), `adjoint` (256 x 256, 8 spp, 3 bounces: forward
vs backward time) and `batch` (the batched workload above); --no-large / --no-adjoint / --no-batch
/ --no-build leave them out.

`value` times the step with its inputs resident in HBM (CUDA events on the launching stream, L2
flushed by a 256 MiB write between timed steps). `e2e` times the same step through the C ABI with
host buffers (trace: the radiance read back into pinned memory every step; build: the records
copied in from pinned memory and the tree header read back). Multi-GPU: replicas (neither the
build nor a 512^2 frame is sharded); every rank runs the same workload, value = the work of all
ranks / the max time over ranks.
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

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "caelix-renderer_b200"))

N_LEAVES = 1 << 22
TRACE_W = TRACE_H = 512
TRACE_BOUNCES = 4
L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0
BUILD_BYTES_PER_LEAF = 492  # emit 112 + Morton 32 + sort 68 + Karras 20 + aggregate 100 + wide 160
# The sort stage of the build: four onesweep passes (pass 0 reads keys only, 12 B; passes 1-3 read
# and write pairs, 16 B).
SORT_STAGE_BYTES_PER_PAIR = 60.0
# The build's dominant stage: the tile kernel and the upper aggregation (aggregation 52 B read +
# 48 B written, 4-wide collapse 96 x 1/2 read + 224 x 1/2 written, per leaf).
TILE_STAGE_BYTES_PER_LEAF = 100.0 + 160.0
TRACE_BYTES_PER_RAY = 64  # lower bound: one hash slot sector + one record sector per ray
# DRAM bytes (read + write) measured by ncu (one capture per kernel, cold cache; profiles/): the sort
# stage at 4,194,304 pairs (a pipelined pass times four), scaled per pair; the tile stage at
# 2,097,152 leaves (lt_tile_kernel + lt_aggregate_upper_kernel), scaled per leaf; the wavefront
# frame of the 512 x 512 trace (trace and shade kernels of its 5 bounce iterations).
SORT_STAGE_DRAM_BYTES_PER_PAIR = 4 * 34.2e6 / 4194304
TILE_STAGE_DRAM_BYTES_PER_LEAF = (236.7e6 + 378.4e6 + 25.4e6 + 3.1e6) / 2097152
TRACE_FRAME_DRAM_BYTES = 134.7e6


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        # NCCL on the GPU box; gloo where no CUDA device is visible (the host-side tests of the
        # multi-rank plumbing).
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    import torch

    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if cuda:
        torch.cuda.synchronize()


def base_line(args, world, metric, value, unit, ms_per_step, config, higher=True):
    return {
        "metric": metric,
        "value": value,
        "unit": unit,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": higher,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config,
    }


TRACE_METRIC = "trace throughput, Mrays/s (primary + bounce + shadow rays counted on the device)"
BATCH_METRIC = "batched trace throughput, Mrays/s (light-tree rebuild + trace of every scene per step)"
FLUSH_METRIC = "incremental scene flush time after a 1% edit (ms)"
def trace_config(world: int) -> dict:
    """The headline workload's config, the same in both arms."""
    return {
        "workload": "plain brick-DDA trace: 128^3-voxel world (16^3 bricks, 30% occupied, value noise seed 2), "
                    "512x512 pinhole, 1 spp, 4 bounces, light-tree NEE with MIS, fp32 radiance",
        "bricks": 1229,
        "emissive_bricks": 12,
        "width": TRACE_W,
        "height": TRACE_H,
        "spp": 1,
        "bounces": TRACE_BOUNCES,
        "l2": "flushed between timed steps (256 MiB write)",
        "parallelism": f"replicas x{world}",
    }


def compact(obj, digits: int = 4):
    """Floats rounded to `digits` significant digits (the detail sections of the line stay short)."""
    if isinstance(obj, float):
        return float(f"{obj:.{digits}g}")
    if isinstance(obj, dict):
        return {k: compact(v, digits) for k, v in obj.items()}
    if isinstance(obj, list):
        return [compact(v, digits) for v in obj]
    return obj

# ---------------------------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle (the reference's shader logic restated in C; the
# reference's own GPU code is HLSL for Vulkan and has no CPU build)


_ORACLE_SCENE = None


def oracle_trace(seconds: float, threads: int, first_seed: int = 1):
    """Renders whole frames of the trace workload with the oracle (seeds first_seed, +1, ...) on
    `threads` threads for about `seconds`; returns (rays, seconds, frames)."""
    global _ORACLE_SCENE
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib
    from caelix_b200 import workloads

    if _ORACLE_SCENE is None:
        _ORACLE_SCENE = oracle_lib.OracleScene(oracle_lib.load(), workloads.noise_world())
    rays = 0
    frames = 0
    t0 = time.perf_counter()
    while frames == 0 or time.perf_counter() - t0 < seconds:
        _, r = _ORACLE_SCENE.render(TRACE_W, TRACE_H, spp=1, bounces=TRACE_BOUNCES, seed=first_seed + frames,
                                    threads=threads)
        rays += int(r.sum())
        frames += 1
    return rays, time.perf_counter() - t0, frames


def oracle_build_throughput(n: int, seconds: float, threads: int):
    """Independent oracle builds of an n-record sample on `threads` host threads for about `seconds`."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib
    from caelix_b200 import workloads

    lib = oracle_lib.load()
    rec, group, frames = workloads.brick_light_records(n, grid_bricks=1024, group_shift=4)
    counts = [0] * threads
    stop = time.perf_counter() + seconds

    def worker(k):
        while time.perf_counter() < stop or counts[k] == 0:
            oracle_lib.lt_build(lib, rec, record_group=group, group_frames=frames)
            counts[k] += 1

    t0 = time.perf_counter()
    ts = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    wall = time.perf_counter() - t0
    return sum(counts) * n / wall / 1e6, sum(counts), wall


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == "build":
        n = 1 << 18
        for _ in range(args.warmup):
            oracle_build_throughput(n, 0.5, threads)
        values = [oracle_build_throughput(n, 4.0, threads)[0] for _ in range(args.steps)]
        value = statistics.mean(values)
        line = base_line(args, args.gpus, "light-tree build throughput (Mleaves/s)", value, "Mleaves/s", None,
                         {"workload": f"light-tree build, {N_LEAVES} brick light records (sampled at {n} per build)"})
        sample = f"independent oracle builds of {n} records on {threads} threads, ~4 s per step"
    elif args.workload == "flush":
        # The oracle has no incremental path: every flush is a whole scene build (records, hash
        # table, light records, light tree) on one thread, timed on a sample of the generator
        # and scaled by brick count to the 2M-brick world.
        sys.path.insert(0, os.path.join(REPO, "tests"))
        import oracle_lib
        from caelix_b200 import workloads

        lib = oracle_lib.load()
        vs = workloads.noise_world(grid_bricks=(48, 48, 24), brick_occupancy=0.476, voxel_fill=0.25,
                                   emissive_fraction=0.05, seed=3)
        for _ in range(min(args.warmup, 1)):
            oracle_lib.OracleScene(lib, vs).close()
        per_step = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            builds = 0
            while builds == 0 or time.perf_counter() - t0 < 2.0:
                oracle_lib.OracleScene(lib, vs).close()
                builds += 1
            per_step.append((time.perf_counter() - t0) / builds)
        value = 1e3 * statistics.mean(per_step) * args.flush_bricks / vs.brick_count
        line = base_line(args, args.gpus, FLUSH_METRIC, value, "ms", value,
                         {"workload": f"scene flush of the 256x256x64-brick world with {args.flush_bricks} occupied "
                                      "bricks (5% emissive)"}, higher=False)
        threads = 1
        sample = (f"whole oracle scene builds of a {vs.brick_count}-brick world of the same generator on one thread "
                  f"(~2 s per step), scaled by brick count to {args.flush_bricks}")
    elif args.workload == "batch":
        # The oracle renders the smallest scene of the batch plan at its viewport, 2 spp, 4 bounces,
        # on every host thread.
        sys.path.insert(0, os.path.join(REPO, "tests"))
        import oracle_lib
        from caelix_b200 import workloads

        plan = workloads.batch_plan(args.batch_scenes)
        i = min(range(len(plan)), key=lambda j: plan[j][0])
        bricks, side = plan[i]
        osc = oracle_lib.OracleScene(oracle_lib.load(), workloads.batch_scene(bricks, seed=100 + i))
        rays = 0
        secs = 0.0
        frames = 0
        for k in range(args.steps):
            t0 = time.perf_counter()
            while True:
                _, r = osc.render(side, side, spp=BATCH_SPP, bounces=BATCH_BOUNCES, seed=1 + k + frames,
                                  threads=threads)
                rays += int(r.sum())
                frames += 1
                if time.perf_counter() - t0 >= 2.0:
                    break
            secs += time.perf_counter() - t0
        value = rays / secs / 1e6
        line = base_line(args, args.gpus, BATCH_METRIC, value, "Mrays/s", 1e3 * secs / frames,
                         {"workload": f"{args.batch_scenes} scenes, brick counts log-uniform in [1k, 500k], square "
                                      f"viewports among 256/512/1024, {BATCH_SPP} spp, {BATCH_BOUNCES} bounces"})
        sample = (f"{frames} oracle renders of the plan's smallest scene ({bricks} bricks, {side}x{side}) on "
                  f"{threads} threads (~2 s per step)")
    else:
        for _ in range(min(args.warmup, 1)):
            oracle_trace(0.0, threads, 5000)
        rays = 0
        secs = 0.0
        frames = 0
        for k in range(args.steps):
            r, s, f = oracle_trace(2.0, threads, 1 + 100 * k)
            rays += r
            secs += s
            frames += f
        value = rays / secs / 1e6
        line = base_line(args, args.gpus, TRACE_METRIC, value, "Mrays/s", 1e3 * secs / frames,
                         trace_config(args.gpus))
        sample = f"{frames} oracle renders of the whole 512x512 frame on {threads} threads (~2 s per step)"
    line["impl"] = "reference"
    line["cpu_baseline"] = {"value": value, "unit": line["unit"], "cores": threads, "kind": "port", "sample": sample}
    line["e2e"] = {"value": value, "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# Our arm


def measure_build(args, world, local, dev, stream, flush, records):
    import numpy as np
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    sptr = stream.cuda_stream
    rec, group, frames = workloads.brick_light_records(records, grid_bricks=1024, group_shift=4)
    n = len(rec)
    d_rec = torch.from_numpy(rec.view(np.uint8)).cuda()
    d_group = torch.from_numpy(group.view(np.int32)).cuda()
    d_frames = torch.from_numpy(frames.view(np.uint8)).cuda()
    bvh = caelix_b200.LightBvh(dev, n)

    def build():
        bvh.build(d_rec, n, record_group=d_group, group_frames=d_frames, group_count=len(frames), stream=sptr)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            build()
    stream.synchronize()
    bvh.stats()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            build()
            stops[k].record(stream)
    stream.synchronize()
    barrier(world)
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(starts, stops)), world) / args.steps
    launches = bvh.stats().kernel_launches * args.steps
    bvh.set_profiling(True)
    stage_ms = np.zeros(7)
    reps = 5
    with torch.cuda.stream(stream):
        for _ in range(reps):
            flush.zero_()
            build()
            stage_ms += np.array(bvh.stats().stage_ms[:])
    stage_ms /= reps
    bvh.set_profiling(False)
    peak, peak_kind = measured_peaks()
    sort_achieved = SORT_STAGE_BYTES_PER_PAIR * n / (stage_ms[2] / 1e3) / 1e9
    tile_achieved = TILE_STAGE_BYTES_PER_LEAF * n / (stage_ms[5] / 1e3) / 1e9
    build_achieved = BUILD_BYTES_PER_LEAF * n / (ms / 1e3) / 1e9

    # The 4,096-record plain build, L2 flushed between builds.
    rec1, _, _ = workloads.brick_light_records(4096)
    d_rec1 = torch.from_numpy(rec1.view(np.uint8)).cuda()
    bvh1 = caelix_b200.LightBvh(dev, 4096)
    c1 = []
    with torch.cuda.stream(stream):
        for k in range(args.warmup + args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bvh1.build(d_rec1, 4096, stream=sptr)
            b.record(stream)
            if k >= args.warmup:
                c1.append((a, b))
    stream.synchronize()
    config1_ms = max_over_ranks(statistics.mean(a.elapsed_time(b) for a, b in c1), world)

    # End to end through the C ABI: records from pinned memory, build, header and state read back.
    h_rec = torch.from_numpy(rec.view(np.uint8)).pin_memory()
    h_group = torch.from_numpy(group.view(np.int32)).pin_memory()
    h_frames = torch.from_numpy(frames.view(np.uint8)).pin_memory()
    e_rec, e_group, e_frames = torch.empty_like(d_rec), torch.empty_like(d_group), torch.empty_like(d_frames)

    def e2e_step():
        with torch.cuda.stream(stream):
            e_rec.copy_(h_rec, non_blocking=True)
            e_group.copy_(h_group, non_blocking=True)
            e_frames.copy_(h_frames, non_blocking=True)
            bvh.build(e_rec, n, record_group=e_group, group_frames=e_frames, group_count=len(frames), stream=sptr)
        return bvh.stats()

    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    e2e_s = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_s += time.perf_counter() - t0
    e2e_ms = max_over_ranks(e2e_s * 1e3, world) / args.steps
    bvh.close()
    bvh1.close()
    # The key figures last: the driver keeps the tail of the line.
    return {
        "workload": f"light-tree build, {n} brick light records in a 1024^3-brick grid (16^3-brick groups)",
        "records": n,
        "stage_ms": {name: float(v) for name, v in zip(
            ["emit_bounds", "morton_hist", "sort_4_passes", "karras", "depth_scan", "tile_aggregate_collapse_upper_aggregate", "upper_collapse_finish"],
            stage_ms)},
        "roofline_sort": {"kernel": "sort: 4 onesweep_pipe_kernel passes", "bound": "hbm",
                          "achieved": sort_achieved, "peak": peak, "unit": "GB/s", "frac": sort_achieved / peak,
                          "traffic": SORT_STAGE_DRAM_BYTES_PER_PAIR * n,
                          "algorithmic_bytes_per_launch": SORT_STAGE_BYTES_PER_PAIR * n},
        "e2e": {"value": world * n / (e2e_ms / 1e3) / 1e6, "unit": "Mleaves/s",
                "h2d_bytes_per_step": rec.nbytes + group.nbytes + frames.nbytes, "d2h_bytes_per_step": 128,
                "ms_per_step": e2e_ms},
        "gpu_launches": launches,
        "roofline": {"kernel": "lt_tile_kernel + lt_aggregate_upper_kernel", "bound": "hbm",
                     "achieved": tile_achieved, "peak": peak, "unit": "GB/s", "frac": tile_achieved / peak,
                     "peak_kind": peak_kind, "traffic": TILE_STAGE_DRAM_BYTES_PER_LEAF * n,
                     "traffic_source": "ncu, both kernels at 2M leaves, per leaf",
                     "algorithmic_bytes_per_launch": TILE_STAGE_BYTES_PER_LEAF * n},
        "roofline_build": {"bound": "hbm", "achieved": build_achieved, "peak": peak, "unit": "GB/s",
                           "frac": build_achieved / peak, "bytes_per_leaf": BUILD_BYTES_PER_LEAF},
        "config1_ms": config1_ms,
        "mleaves_per_s": world * n / (ms / 1e3) / 1e6,
        "build_ms": ms,
    }


def measure_trace(args, world, local, dev, stream, flush):
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    sptr = stream.cuda_stream
    vs = workloads.noise_world()
    scene = caelix_b200.Scene.from_voxel_scene(dev, vs)
    renderer = caelix_b200.Renderer(dev, scene)
    out = torch.zeros(TRACE_W * TRACE_H * 3, dtype=torch.float32, device="cuda")

    def render(seed):
        renderer.render(out, TRACE_W, TRACE_H, vs.camera, bounces=TRACE_BOUNCES, seed=seed, spp=1, stream=sptr)

    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            render(1000 + k)
    stream.synchronize()
    rays = 0
    launches = 0
    total_ms = 0.0
    barrier(world)
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                render(1 + k)
                b.record(stream)
            st = renderer.stats()  # waits for the step; outside its events
            rays += st.primary_rays + st.bounce_rays + st.shadow_rays
            launches += st.kernel_launches
            total_ms += a.elapsed_time(b)
    barrier(world)
    ms = max_over_ranks(total_ms, world) / args.steps
    rays_per_step = rays / args.steps
    value = world * rays_per_step / (ms / 1e3) / 1e6

    # End to end through the C ABI, as a host that streams frames would run it: every step renders
    # into one of two device images and reads it back into pinned host memory on a copy stream, so
    # the read-back of step k overlaps the render of step k + 1; the timed region is the wall time
    # of all steps, from the first call to the last image on the host.
    outs = [out, torch.zeros_like(out)]
    hosts = [torch.empty(TRACE_W * TRACE_H * 3, dtype=torch.float32).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    rendered = [torch.cuda.Event() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(count, first_seed):
        for k in range(count):
            i = k & 1
            with torch.cuda.stream(stream):
                if k >= 2:
                    stream.wait_event(copied[i])  # the image's previous read-back is done
                flush.zero_()  # L2 flushed between steps (inside the timed region here)
                renderer.render(outs[i], TRACE_W, TRACE_H, vs.camera, bounces=TRACE_BOUNCES, seed=first_seed + k,
                                spp=1, stream=sptr)
                rendered[i].record(stream)
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(rendered[i])
                hosts[i].copy_(outs[i], non_blocking=True)
                copied[i].record(copy_stream)
        copy_stream.synchronize()
        stream.synchronize()

    e2e_steps(max(args.warmup, 2), 2000)
    flush.zero_()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    e2e_steps(args.steps, 1)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, world) / args.steps
    peak, peak_kind = measured_peaks()
    achieved = TRACE_BYTES_PER_RAY * rays_per_step / (ms / 1e3) / 1e9
    result = {
        "value": value,
        "ms_per_step": ms,
        "rays_per_step": rays_per_step,
        "roofline": {"kernel": "wave_trace_kernel + wave_shade_kernel (the frame)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": TRACE_FRAME_DRAM_BYTES,
                     "traffic_source": "ncu launch list: DRAM bytes of one frame's wave kernels (cold cache)",
                     "bytes_per_ray": TRACE_BYTES_PER_RAY,
                     "note": "latency-bound ray traversal; the bytes are a per-ray lower bound"},
        "e2e": {"value": world * rays_per_step / (e2e_ms / 1e3) / 1e6, "unit": "Mrays/s",
                "h2d_bytes_per_step": 208 + 32, "d2h_bytes_per_step": TRACE_W * TRACE_H * 12, "ms_per_step": e2e_ms,
                "note": "wall time of all steps (L2 flush included); step k's read-back overlaps step k+1's "
                        "render (two images)"},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    renderer.close()
    scene.close()
    return result


def measure_entities(args, world, local, dev, stream, flush, counts=(0, 4, 16, 64)):
    """The cost of entities on the plain trace: the 128^3 world with `n` entities of 2 x 2 x 2
    bricks each (value noise) at seeded positions inside the world and rotations, the same
    512 x 512, 1 spp, 4 bounces frame; each count twice: with half of the entities' bricks emitting
    (their lights join the light trees) and with none emitting (the entities only add geometry).
    Rays meet the entities through the entity BVH after the world's bricks. One flush per run
    (entity bricks, views, light sets), then frames timed with CUDA events."""
    import numpy as np
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    sptr = stream.cuda_stream
    vs = workloads.noise_world()
    out = torch.zeros(TRACE_W * TRACE_H * 3, dtype=torch.float32, device="cuda")
    result = {"workload": "128^3 world + n entities of 2x2x2 bricks (half of their bricks emitting, or none), "
                          "512x512, 1 spp, 4 bounces", "runs": []}
    for n, lit in [(c, l) for c in counts for l in ((True,) if c == 0 else (True, False))]:
        scene = caelix_b200.Scene.from_voxel_scene(dev, vs)
        rng = np.random.default_rng(17)  # the same entities lit and unlit
        for i in range(n):
            ent = workloads.noise_world(grid_bricks=(2, 2, 2), brick_occupancy=1.0, voxel_fill=0.5,
                                        emissive_fraction=0.0, seed=100 + i)
            q = rng.normal(size=4)
            e = scene.add_entity(tuple(rng.uniform(8.0, 112.0, 3)), tuple(q / np.linalg.norm(q)))
            scene.upload_bricks(ent.keys, ent.voxels, entity=e)
            power = np.where(rng.random(ent.brick_count) < 0.5, rng.lognormal(0.0, 1.0, ent.brick_count), 0.0)
            scene.set_brick_power(ent.keys, (power if lit else 0.0 * power).astype(np.float32), entity=e)
        t0 = time.perf_counter()
        scene.flush(sptr)
        flush_s = time.perf_counter() - t0
        renderer = caelix_b200.Renderer(dev, scene)
        with torch.cuda.stream(stream):
            for k in range(max(args.warmup, 1)):
                renderer.render(out, TRACE_W, TRACE_H, vs.camera, bounces=TRACE_BOUNCES, seed=1000 + k, spp=1,
                                stream=sptr)
        stream.synchronize()
        steps = max(1, min(args.steps, 5))
        total_ms, rays = 0.0, 0
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                renderer.render(out, TRACE_W, TRACE_H, vs.camera, bounces=TRACE_BOUNCES, seed=1 + k, spp=1, stream=sptr)
                b.record(stream)
            st = renderer.stats()
            rays += st.primary_rays + st.bounce_rays + st.shadow_rays
            total_ms += a.elapsed_time(b)
        ms = max_over_ranks(total_ms, world) / steps
        result["runs"].append({"entities": n, "lit": lit, "ms_per_frame": ms, "rays_per_frame": rays / steps,
                               "mrays_per_s": world * rays / steps / (ms / 1e3) / 1e6, "flush_wall_s": flush_s})
        renderer.close()
        scene.close()
    return result


def measure_large(args, world, local, dev, stream, flush, rank):
    """The large scene: 2048 x 2048 x 512 voxels (256 x 256 x 64 bricks), ~2M occupied bricks (12 %
    voxel occupancy overall), ~100k emissive bricks; the flush (records, hash table, light records,
    a full light-tree rebuild) and 1920 x 1080 frames at 4 spp, 6 bounces, light-tree NEE; then a
    light-tree-only flush and the flush after re-uploading 1 % of the bricks."""
    import numpy as np
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    t0 = time.perf_counter()
    vs = workloads.noise_world_large()
    gen_s = time.perf_counter() - t0
    scene = caelix_b200.Scene.for_voxel_scene(dev, vs)
    t0 = time.perf_counter()
    scene.upload_bricks(vs.keys, vs.voxels)
    em = vs.power > 0
    scene.set_brick_power(vs.keys, vs.power)
    upload_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    scene.flush(stream.cuda_stream)
    flush_wall_s = time.perf_counter() - t0
    ls = scene.light_stats()
    renderer = caelix_b200.Renderer(dev, scene)
    w, h, spp, bounces = 1920, 1080, 4, 6
    out = torch.zeros(w * h * 3, dtype=torch.float32, device="cuda")
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        renderer.render(out, w, h, vs.camera, bounces=bounces, seed=999, spp=spp, stream=sptr)
    stream.synchronize()
    steps = max(1, min(args.steps, 3))
    rays = 0
    total_ms = 0.0
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            renderer.render(out, w, h, vs.camera, bounces=bounces, seed=1 + 4 * k, spp=spp, stream=sptr)
            b.record(stream)
        st = renderer.stats()
        rays += st.primary_rays + st.bounce_rays + st.shadow_rays
        total_ms += a.elapsed_time(b)
    ms = max_over_ranks(total_ms, world) / steps
    t = renderer.timings()
    # A light-options change that keeps the light codes: the next flush rebuilds only the light tree.
    scene.set_light_options(True, 0.25)
    scene.flush(sptr)
    tree_flush_ms = float(renderer.timings().flush_ms)
    # An edit: 1 % of the bricks uploaded again (to the device staging), then the full flush from
    # the staged bricks (device sort and gather of all bricks, records, hash table, light records).
    # The first such flush also allocates the second light heap and the edit buffers; the second
    # one is the steady state.
    edit_ms = []
    for k in range(2):
        edit = np.random.default_rng(5 + k).choice(vs.brick_count, size=vs.brick_count // 100, replace=False)
        t0 = time.perf_counter()
        scene.upload_bricks(vs.keys[edit], vs.voxels[edit])
        edit_upload_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        scene.flush(sptr)
        edit_flush_wall_s = time.perf_counter() - t0
        edit_ms.append(float(renderer.timings().flush_ms))
    first_edit_flush_ms, edit_flush_ms = edit_ms
    result = {
        "workload": "2048x2048x512-voxel world (256x256x64 bricks), value noise seed 3, 1920x1080, 4 spp, "
                    "6 bounces, light-tree NEE with MIS",
        "bricks": int(vs.brick_count),
        "brick_occupancy": float(vs.brick_count) / (256 * 256 * 64),
        "voxel_occupancy": float((vs.voxels != 0).sum()) / (2048 * 2048 * 512),
        "emissive_bricks": int(em.sum()),
        "light_tree_leaves": int(ls.tree_leaves[0]),
        "light_tree_nodes": int(ls.tree_nodes[0]),
        "flush_ms": float(t.flush_ms),
        "flush_wall_s": flush_wall_s,
        "light_tree_flush_ms": tree_flush_ms,
        "edit_bricks": int(len(edit)),
        "edit_upload_s": edit_upload_s,
        "first_edit_flush_ms": first_edit_flush_ms,
        "edit_flush_ms": edit_flush_ms,
        "edit_flush_wall_s": edit_flush_wall_s,
        "generate_s": gen_s,
        "upload_s": upload_s,
        "frame_ms": ms,
        "rays_per_frame": rays / steps,
        "mrays_per_s": world * rays / steps / (ms / 1e3) / 1e6,
    }
    peak, peak_kind = measured_peaks()
    achieved = TRACE_BYTES_PER_RAY * (rays / steps) / (ms / 1e3) / 1e9
    result["roofline"] = {"kernel": "wave_trace_kernel + wave_shade_kernel (the frame)", "bound": "hbm",
                          "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                          "peak_kind": peak_kind, "traffic": None, "bytes_per_ray": TRACE_BYTES_PER_RAY,
                          "note": "latency-bound ray traversal; the bytes are a per-ray lower bound"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # The oracle's trace over the flushed tables (the light tree its own build), on every host
        # core, over a centred pixel window of the same frame; rays counted by the oracle.
        sys.path.insert(0, os.path.join(REPO, "tests"))
        import oracle_lib

        tab = oracle_lib.TablesScene(oracle_lib.load(), vs, scene.view())
        threads = os.cpu_count() or 1
        ww, wh = 96, 64
        window = ((w - ww) // 2, (h - wh) // 2, (w + ww) // 2, (h + wh) // 2)
        t0 = time.perf_counter()
        _, orays = tab.render(w, h, spp=spp, bounces=bounces, seed=1, window=window, threads=threads)
        cpu_s = time.perf_counter() - t0
        tab.close()
        result["cpu_baseline"] = {"value": float(orays.sum()) / cpu_s / 1e6, "unit": "Mrays/s", "cores": threads,
                                  "kind": "port", "sample": f"oracle trace of a centred {ww}x{wh} window, same frame"}
    renderer.close()
    scene.close()
    return result


# Algorithmic bytes per brick of a full flush: slot sort (12 + 4 + 68), gather (1040 read + 1040
# write), hash build (~150), finalize (1024 + 6 x 128 faces read, 1096 written).
FLUSH_BYTES_PER_BRICK = 84 + 2080 + 150 + 2888


def measure_flush(args, world, local, dev, stream):
    """The scene flush on the large world (`--flush-bricks` occupied bricks of the 256 x 256 x 64
    brick grid, 5 % of them emissive): the first flush after the upload (a full build from the
    device staging: slot sort and gather, hash table, bitmap, records, light records, light tree);
    per step an edit of 1 % of the bricks (their values uploaded again) and its flush (incremental:
    the edited bricks and their neighbours finalized again, light records and light tree rebuilt);
    then a light-options change (the light tree alone) and a full rebuild (a new brick). The bricks
    are loaded from a .cxw world file written from the generated world (its read, decode and upload
    timed as `world_file`)."""
    import numpy as np

    import caelix_b200
    from caelix_b200 import workloads

    import tempfile

    from caelix_b200 import cxw

    nb = args.flush_bricks
    vs = workloads.noise_world_large(occupied_bricks=nb, emissive_bricks=max(1, nb // 20))
    scene = caelix_b200.Scene.for_voxel_scene(dev, vs)
    renderer = caelix_b200.Renderer(dev, scene)
    sptr = stream.cuda_stream
    # The bricks arrive from a .cxw world file: read, decoded on every host thread, uploaded.
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "world.cxw")
        t0 = time.perf_counter()
        data = cxw.from_voxel_scene(vs)
        with open(path, "wb") as fh:
            fh.write(data)
        write_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        wfile = caelix_b200.WorldFile(path)
        open_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        origin, loaded = wfile.upload_entity(0, scene)
        upload_s = time.perf_counter() - t0
        wfile.close()
    # The reader drops all-air bricks; the scene holds the others, moved to the returned origin.
    keep = (vs.voxels != 0).any(axis=1)
    assert loaded == int(keep.sum())
    keys = vs.keys[keep] - np.array(origin, np.int32)
    voxels, power = vs.voxels[keep], vs.power[keep]
    threads = os.cpu_count() or 1
    em = power > 0
    scene.set_brick_power(keys, power)
    scene.flush(sptr)
    first_ms = float(renderer.timings().flush_ms)
    rng = np.random.default_rng(5)
    edit_ms, edit_upload_s = [], []
    for k in range(args.warmup + args.steps):
        edit = rng.choice(len(keys), size=max(1, len(keys) // 100), replace=False)
        t0 = time.perf_counter()
        scene.upload_bricks(keys[edit], voxels[edit])
        up = time.perf_counter() - t0
        scene.flush(sptr)
        if k >= args.warmup:
            edit_ms.append(float(renderer.timings().flush_ms))
            edit_upload_s.append(up)
    scene.set_light_options(True, 0.25)
    scene.flush(sptr)
    tree_ms = float(renderer.timings().flush_ms)
    # A brick at the first free cell of the grid: the key set changes, so the flush rebuilds all.
    gx, gy, gz = (int(v) for v in keys.max(axis=0) + 1)
    lin = keys[:, 0].astype(np.int64) + gx * (keys[:, 1] + gy * keys[:, 2].astype(np.int64))
    free = np.setdiff1d(np.arange(min(gx * gy * gz, len(lin) + 1)), lin)[0]
    key = np.array([[free % gx, (free // gx) % gy, free // (gx * gy)]], np.int32)
    scene.upload_bricks(key, np.full((1, 512), 0x8001, np.uint16))
    scene.flush(sptr)
    full_ms = float(renderer.timings().flush_ms)
    renderer.close()
    scene.close()
    ms = max_over_ranks(float(np.mean(edit_ms)), world)
    full = max_over_ranks(full_ms, world)
    achieved = len(keys) * FLUSH_BYTES_PER_BRICK / (full / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    return {
        "workload": f"scene flush of the 256x256x64-brick world with {len(keys)} occupied bricks "
                    f"({int(em.sum())} emissive): incremental flush after re-uploading 1% of the bricks",
        "bricks": int(len(keys)),
        "edit_bricks": int(max(1, len(keys) // 100)),
        "edit_flush_ms": ms,
        "edit_upload_s": float(np.mean(edit_upload_s)),
        "first_flush_ms": first_ms,
        "full_rebuild_ms": full,
        "light_tree_flush_ms": tree_ms,
        "world_file": {"bytes": len(data), "write_s": write_s, "open_s": open_s,
                       "decode_upload_s": upload_s, "bricks": int(loaded), "host_threads": threads,
                       "mbricks_per_s": loaded / upload_s / 1e6,
                       "note": "caelix_world_open + caelix_world_upload_entity (raw inflate and decode on every "
                               "host thread, then caelix_scene_upload_bricks per sector)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "kernel": f"the full rebuild ({FLUSH_BYTES_PER_BRICK} algorithmic bytes per brick)"},
    }


ADJ_W = ADJ_H = 256
ADJ_SPP = 8
ADJ_BOUNCES = 3


def measure_adjoint(args, world, local, dev, stream, flush, rank):
    """The differentiation workload: the solid-brick world of the plain light-tree build (4096 brick
    records, 32^3 brick grid), 256 x 256, 8 spp, 3 bounces; L2 loss against a target rendered with
    albedo and power perturbed by up to 10 %. Times caelix_renderer_render (forward) and
    caelix_renderer_backward (dL/dalbedo 128 x 3 and dL/dpower per brick, path replay) with CUDA
    events, L2 flushed before each; the CPU baseline is the double-precision adjoint reference
    (the oracle, all host threads)."""
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    sptr = stream.cuda_stream
    vs = workloads.solid_brick_scene()
    scene = caelix_b200.Scene.from_voxel_scene(dev, vs)
    tscene = caelix_b200.Scene.from_voxel_scene(dev, workloads.perturbed(vs))
    r = caelix_b200.Renderer(dev, scene)
    tr = caelix_b200.Renderer(dev, tscene)
    img = torch.zeros(ADJ_W * ADJ_H * 3, device="cuda")
    tgt = torch.zeros_like(img)
    d_alb = torch.zeros(65536 * 3, device="cuda")
    d_pow = torch.zeros(vs.brick_count, device="cuda")

    def forward():
        r.render(img, ADJ_W, ADJ_H, vs.camera, bounces=ADJ_BOUNCES, seed=1, spp=ADJ_SPP, stream=sptr)

    def backward():
        r.backward(d_rad, ADJ_W, ADJ_H, vs.camera, d_alb, d_pow, bounces=ADJ_BOUNCES, seed=1, spp=ADJ_SPP,
                   stream=sptr)

    with torch.cuda.stream(stream):
        tr.render(tgt, ADJ_W, ADJ_H, vs.camera, bounces=ADJ_BOUNCES, seed=1, spp=ADJ_SPP, stream=sptr)
        forward()
        d_rad = 2.0 * (img - tgt)
    stream.synchronize()

    def timed(fn, steps):
        total = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total / steps

    for _ in range(args.warmup):
        forward()
        backward()
    stream.synchronize()
    steps = max(1, min(args.steps, 10))
    fwd_ms = max_over_ranks(timed(forward, steps), world)
    st = r.stats()
    fwd_rays = st.primary_rays + st.bounce_rays + st.shadow_rays
    bwd_ms = max_over_ranks(timed(backward, steps), world)
    result = {
        "workload": f"solid-brick world of the 4096-record build (32^3 bricks), {ADJ_W}x{ADJ_H}, {ADJ_SPP} spp, "
                    f"{ADJ_BOUNCES} bounces, L2 loss vs a target with albedo/power perturbed by up to 10%; "
                    "gradients w.r.t. the albedo table (65536 codes x 3) and per-brick power (path replay, sampling held fixed)",
        "bricks": int(vs.brick_count),
        "forward_ms": fwd_ms,
        "backward_ms": bwd_ms,
        "adjoint_over_forward": bwd_ms / fwd_ms,
        "forward_mrays_per_s": fwd_rays / (fwd_ms / 1e3) / 1e6,
        "parity": "tests/test_adjoint_gpu.py: vs the double-precision reference and central differences (1e-3)",
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "tests"))
        import oracle_lib

        osc = oracle_lib.OracleScene(oracle_lib.load(), vs)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        osc.adjoint(ADJ_W, ADJ_H, spp=ADJ_SPP, bounces=ADJ_BOUNCES, seed=1, d_radiance=d_rad.cpu().numpy(),
                    threads=threads)
        cpu_s = time.perf_counter() - t0
        osc.close()
        result["cpu_baseline"] = {"value": cpu_s * 1e3, "unit": "ms", "cores": threads, "kind": "port",
                                  "sample": "one double-precision adjoint of the whole frame (oracle oc_adjoint), "
                                            f"{threads} threads"}
    r.close()
    tr.close()
    scene.close()
    tscene.close()
    return result


BATCH_SPP = 2
BATCH_BOUNCES = 4
TUNE_CACHE = os.path.join(REPO, "caelix-renderer_b200", "tuning", "batch_tuning.json")


def measure_batch(args, world, local, dev, stream):
    """The batched workload: `--batch-scenes` scenes (brick counts log-uniform in [1k, 500k], 1 %
    emissive, the plain scene's generator), square viewports uniform among 256, 512, 1024, 2 spp,
    4 bounces, light-tree NEE. One step = every scene's light-tree rebuild and the trace of every
    view. Timed three ways on the same scenes, renderers and targets (CUDA events around a step):
      batched     caelix_batch_run: one CUDA graph launch (parallel light-tree builds, then one
                  persistent trace launch over all views), launch parameters from the autotuner;
      sequential  one scene at a time through the plain C ABI: caelix_scene_set_light_options +
                  caelix_scene_flush (the light-tree rebuild and its status read-back) +
                  caelix_renderer_render, 64 times;
      per-view    the batched graph of one view, 64 times (separates the kernel from the batching).
    The scenes (~10 GB on the device) are larger than L2, so no flush is needed between steps."""
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    sptr = stream.cuda_stream
    plan = workloads.batch_plan(args.batch_scenes)
    t0 = time.perf_counter()
    scenes, renderers, views = [], [], []
    bricks = lights = 0
    for i, (count, side) in enumerate(plan):
        vs = workloads.batch_scene(count, seed=100 + i)
        scene = caelix_b200.Scene.from_voxel_scene(dev, vs)
        renderer = caelix_b200.Renderer(dev, scene)
        out = torch.zeros(side * side * 3, dtype=torch.float32, device="cuda")
        views.append((renderer, out, side, side, vs.camera, BATCH_BOUNCES, 1 + i, BATCH_SPP))
        scenes.append(scene)
        renderers.append(renderer)
        bricks += vs.brick_count
        lights += scene.view().light_count
        del vs
    setup_s = time.perf_counter() - t0
    torch.cuda.synchronize()

    def timed(step, steps):
        total_ms = 0.0
        for k in range(steps):
            with torch.cuda.stream(stream):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                step(k)
                b.record(stream)
            b.synchronize()
            total_ms += a.elapsed_time(b)
        return total_ms / steps

    steps = max(1, min(args.steps, 5))
    batch = caelix_b200.Batch(dev, views, rebuild_light_trees=True)
    t0 = time.perf_counter()
    if args.tuning:
        batch.set_tuning(**{k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))})
        tuning = batch.tuning()
    else:
        tuning = batch.autotune(args.tune_cache, repeats=2, stream=sptr)
    tune_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        batch.run(sptr)
    stream.synchronize()
    barrier(world)
    with ClockSampler(local) as clocks:
        batched_ms = timed(lambda k: batch.run(sptr), steps)
    barrier(world)
    batched_ms = max_over_ranks(batched_ms, world)
    st = batch.stats()
    rays = st.primary_rays + st.bounce_rays + st.shadow_rays

    def sequential(k):
        for scene, (renderer, out, w, h, cam, bounces, seed, spp) in zip(scenes, views):
            scene.set_light_options(True)
            scene.flush(sptr)
            renderer.render(out, w, h, cam, bounces=bounces, seed=seed, spp=spp, stream=sptr)

    for _ in range(max(1, args.warmup // 2)):
        sequential(0)
    stream.synchronize()
    sequential_ms = max_over_ranks(timed(sequential, steps), world)
    seq_rays = 0
    for r in renderers:
        rs = r.stats()
        seq_rays += rs.primary_rays + rs.bounce_rays + rs.shadow_rays

    singles = []
    for v in views:
        b1 = caelix_b200.Batch(dev, [v], rebuild_light_trees=True)
        b1.set_tuning(**{k: val for k, val in tuning.as_dict().items()})
        b1.run(sptr)
        singles.append(b1)
    stream.synchronize()
    per_view_ms = max_over_ranks(timed(lambda k: [b1.run(sptr) for b1 in singles], steps), world)
    for b1 in singles:
        b1.close()

    result = {
        "workload": f"{len(plan)} scenes, brick counts log-uniform in [1k, 500k] (1% emissive), square viewports "
                    f"uniform among 256/512/1024, {BATCH_SPP} spp, {BATCH_BOUNCES} bounces, light-tree rebuild + "
                    "trace per scene per step",
        "scenes": len(plan),
        "bricks": int(bricks),
        "light_tree_leaves": int(lights),
        "pixels": int(sum(v[2] * v[3] for v in views)),
        "setup_s": setup_s,
        "autotune_s": tune_s,
        "tuning": tuning.as_dict(),
        "graph_kernel_nodes": int(st.kernel_launches),
        "wavefront": int(st.wavefront),
        "rays_per_step": int(rays),
        "sequential_rays_per_step": int(seq_rays),
        "batched_ms": batched_ms,
        "sequential_ms": sequential_ms,
        "per_view_batched_ms": per_view_ms,
        "speedup_vs_sequential": sequential_ms / batched_ms,
        "batched_mrays_per_s": world * rays / (batched_ms / 1e3) / 1e6,
        "sequential_mrays_per_s": world * seq_rays / (sequential_ms / 1e3) / 1e6,
        "clocks": clocks.summary(),
    }
    batch.close()
    for r in renderers:
        r.close()
    for s in scenes:
        s.close()
    return result


def run_ours(args, world, rank, local):
    import torch

    import caelix_b200

    torch.cuda.set_device(local)
    dev = caelix_b200.Device(local)
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    if args.workload == "batch":
        batch = measure_batch(args, world, local, dev, stream)
        line = base_line(args, world, BATCH_METRIC, batch["batched_mrays_per_s"], "Mrays/s", batch["batched_ms"],
                         {"workload": batch["workload"], "scenes": batch["scenes"], "spp": BATCH_SPP,
                          "bounces": BATCH_BOUNCES, "l2": "inputs larger than L2 (~10 GB of scenes)",
                          "parallelism": f"replicas x{world}"})
        line["batch"] = batch
        line["gpu_launches"] = args.steps * batch["graph_kernel_nodes"]
        line["clocks"] = batch["clocks"]
        if rank == 0:
            print(json.dumps(line), flush=True)
        dev.close()
        return
    if args.workload == "flush":
        fl = measure_flush(args, world, local, dev, stream)
        line = base_line(args, world, FLUSH_METRIC, fl["edit_flush_ms"], "ms",
                         fl["edit_flush_ms"], {"workload": fl["workload"], "bricks": fl["bricks"],
                                               "l2": "inputs larger than L2 (2 GB of bricks)",
                                               "parallelism": f"replicas x{world}"}, higher=False)
        line["flush"] = fl
        line["roofline"] = fl["roofline"]
        if rank == 0:
            print(json.dumps(line), flush=True)
        dev.close()
        return
    build = None if args.no_build else measure_build(args, world, local, dev, stream, flush, args.records)
    if args.workload == "build":
        line = base_line(args, world, "light-tree build throughput (Mleaves/s)", build["mleaves_per_s"], "Mleaves/s",
                         build["build_ms"], {"workload": build["workload"], "records": build["records"],
                                             "l2": "flushed between timed steps (256 MiB write)",
                                             "parallelism": f"replicas x{world}"})
        line.update({k: build[k] for k in ("roofline", "roofline_sort", "roofline_build", "e2e", "gpu_launches",
                                           "stage_ms", "config1_ms")})
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            v, builds, wall = oracle_build_throughput(1 << 20, 10.0, 1)
            line["cpu_baseline"] = {"value": v, "unit": "Mleaves/s", "cores": 1, "kind": "port",
                                    "sample": f"{builds} oracle builds of 1048576 records, 1 thread, {wall:.1f} s"}
    else:
        trace = measure_trace(args, world, local, dev, stream, flush)
        line = base_line(args, world, TRACE_METRIC, trace["value"], "Mrays/s", trace["ms_per_step"],
                         trace_config(world))
        line.update({k: trace[k] for k in ("roofline", "e2e", "gpu_launches", "clocks", "rays_per_step")})
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            rays, secs, frames = oracle_trace(10.0, 1)
            line["cpu_baseline"] = {"value": rays / secs / 1e6, "unit": "Mrays/s", "cores": 1, "kind": "port",
                                    "sample": f"{frames} oracle renders of the whole 512x512 frame, 1 thread, "
                                              f"{secs:.1f} s"}
        # The detail sections, rounded; the build goes last, so that the end of the line holds it.
        if args.large:
            line["large"] = compact(measure_large(args, world, local, dev, stream, flush, rank))
        if args.adjoint:
            line["adjoint"] = compact(measure_adjoint(args, world, local, dev, stream, flush, rank))
        if args.entities:
            line["entities"] = compact(measure_entities(args, world, local, dev, stream, flush))
        if args.batch:
            line["batch"] = compact(measure_batch(args, world, local, dev, stream))
        if build is not None:
            # The key figures at the very end of the line (the driver keeps its tail).
            section = {k: build[k] for k in ("records", "stage_ms", "e2e")}
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                v, builds, wall = oracle_build_throughput(1 << 18, 8.0, 1)
                section["cpu_baseline"] = {"value": v, "unit": "Mleaves/s", "cores": 1, "kind": "port",
                                           "sample": f"{builds} oracle builds of 262144 records, 1 thread"}
            section.update({k: build[k] for k in ("roofline", "roofline_build", "config1_ms", "mleaves_per_s",
                                                  "build_ms")})
            for k in ("traffic_source", "peak_kind"):
                section["roofline"].pop(k, None)
            line["build"] = compact(section)
    if rank == 0:
        print(json.dumps(line), flush=True)
    dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["trace", "build", "batch", "flush"], default="trace")
    ap.add_argument("--flush-bricks", type=int, default=2_000_000, help="occupied bricks of the flush workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--records", type=int, default=N_LEAVES, help="records of the build workload")
    ap.add_argument("--no-build", action="store_true", help="trace workload only: skip the build section")
    ap.add_argument("--large", action=argparse.BooleanOptionalAction, default=True,
                    help="add the large-scene section (2M bricks, 1080p, 4 spp, 6 bounces)")
    ap.add_argument("--batch", action=argparse.BooleanOptionalAction, default=True,
                    help="add the batched section (64 scenes: batched graph vs one scene at a time)")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--adjoint", action=argparse.BooleanOptionalAction, default=True,
                    help="add the differentiation section (forward vs backward time)")
    ap.add_argument("--entities", action=argparse.BooleanOptionalAction, default=True,
                    help="add the entities section (the trace with 4, 16 and 64 lit entities)")
    ap.add_argument("--tune-cache", default=TUNE_CACHE, help="the autotuner's JSON cache (read, and written on a miss)")
    ap.add_argument("--tuning", default="", help="fixed batch tuning instead of the autotuner, e.g. "
                    "min_blocks=8,block_width=8,refill_min=4")
    args = ap.parse_args()
    world, rank, local = dist_setup()
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
