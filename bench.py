#!/usr/bin/env python3
"""Benchmark of the scene-flush / trace hot path on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (seeded synthetic inputs with the shapes of the benchmark configurations; no dataset):
  build   the light-tree build over N_LEAVES brick light records (brick coords uniform in a
          1024^3-brick grid, render groups of 16^3 bricks with identity frames, power
          log-normal(0, 1) split over the faces): gather emit, centre bounds, Morton codes, onesweep
          radix sort, Karras, aggregation, depth + scan, 4-wide collapse. value = Mleaves/s.
          The 4,096-record plain build is timed beside it (config1_ms).

A step is one pass of the hot path over one batch of inputs already resident in HBM (`value`);
`e2e` times the same step through the C ABI with the inputs copied from pinned host memory and the
tree header read back, every step. Multi-GPU: replicas (the build does not shard); every rank runs
the same workload, value = the work of all ranks / the max time over ranks.
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
L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0
BUILD_BYTES_PER_LEAF = 492  # emit 112 + Morton 32 + sort 68 + Karras 20 + aggregate 100 + wide 160
SORT_PASS_BYTES_PER_PAIR = 60.0 / 4  # pass 0 reads keys only (12 B), passes 1-3 read and write pairs (16 B)


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

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    import torch

    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


# ---------------------------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle (the reference's build restated in C; the reference's
# GPU code is HLSL for Vulkan and cannot run here)


def oracle_build_throughput(n: int, seconds: float, threads: int):
    """Runs independent oracle builds of an n-record sample on `threads` host threads for about
    `seconds`; returns (Mleaves/s, builds, wall seconds)."""
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
    builds = sum(counts)
    return builds * n / wall / 1e6, builds, wall


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = 1 << 18
    values = []
    for _ in range(args.warmup):
        oracle_build_throughput(n, 0.5, threads)
    for _ in range(args.steps):
        v, builds, wall = oracle_build_throughput(n, 4.0, threads)
        values.append(v)
    value = statistics.mean(values)
    line = {
        "impl": "reference",
        "metric": "light-tree build throughput (Mleaves/s)",
        "value": value,
        "unit": "Mleaves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"light-tree build, {N_LEAVES} brick light records (sampled at {n} per build)",
                   "records": N_LEAVES},
        "cpu_baseline": {"value": value, "unit": "Mleaves/s", "cores": threads, "kind": "port",
                         "sample": f"independent oracle builds of {n} records on {threads} threads, ~4 s per step"},
        "e2e": {"value": value, "unit": "Mleaves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# Our arm


def run_build(args, world, rank, local):
    import numpy as np
    import torch

    import caelix_b200
    from caelix_b200 import workloads

    torch.cuda.set_device(local)
    dev = caelix_b200.Device(local)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    rec, group, frames = workloads.brick_light_records(args.records, grid_bricks=1024, group_shift=4)
    n = len(rec)
    d_rec = torch.from_numpy(rec.view(np.uint8)).cuda()
    d_group = torch.from_numpy(group.view(np.int32)).cuda()
    d_frames = torch.from_numpy(frames.view(np.uint8)).cuda()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    bvh = caelix_b200.LightBvh(dev, n)

    def build():
        bvh.build(d_rec, n, record_group=d_group, group_frames=d_frames, group_count=len(frames), stream=sptr)

    # Warm-up.
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            build()
    stream.synchronize()
    bvh.stats()

    # Timed region: K builds, L2 flushed between them (outside the events), events on the stream.
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                build()
                stops[k].record(stream)
        stream.synchronize()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, stops)]
    total_ms = max_over_ranks(sum(step_ms), world)
    ms_per_step = total_ms / args.steps
    value = world * n / (ms_per_step / 1e3) / 1e6
    stats = bvh.stats()
    launches = stats.kernel_launches * args.steps

    # Per-stage timing of one build (profiling events) for the roofline of the dominant kernel.
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
    sort_pass_ms = stage_ms[2] / 4
    peak, peak_kind = measured_peaks()
    sort_achieved = SORT_PASS_BYTES_PER_PAIR * n / (sort_pass_ms / 1e3) / 1e9
    build_achieved = BUILD_BYTES_PER_LEAF * n / (ms_per_step / 1e3) / 1e9

    # The plain 4,096-record build (config 1), L2 flushed between builds.
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

    # End to end through the C ABI: pinned host records -> device, build, tree header and state read
    # back by caelix_light_bvh_get_stats (which waits for the build), every step; host clock per step.
    h_rec = torch.from_numpy(rec.view(np.uint8)).pin_memory()
    h_group = torch.from_numpy(group.view(np.int32)).pin_memory()
    h_frames = torch.from_numpy(frames.view(np.uint8)).pin_memory()
    e2e_dev_rec = torch.empty_like(d_rec)
    e2e_dev_group = torch.empty_like(d_group)
    e2e_dev_frames = torch.empty_like(d_frames)

    def e2e_step():
        with torch.cuda.stream(stream):
            e2e_dev_rec.copy_(h_rec, non_blocking=True)
            e2e_dev_group.copy_(h_group, non_blocking=True)
            e2e_dev_frames.copy_(h_frames, non_blocking=True)
            bvh.build(e2e_dev_rec, n, record_group=e2e_dev_group, group_frames=e2e_dev_frames,
                      group_count=len(frames), stream=sptr)
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
    e2e_value = world * n / (e2e_ms / 1e3) / 1e6
    h2d = rec.nbytes + group.nbytes + frames.nbytes

    line = {
        "metric": "light-tree build throughput (Mleaves/s)",
        "value": value,
        "unit": "Mleaves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"light-tree build, {n} brick light records in a 1024^3-brick grid (16^3-brick groups)",
            "records": n,
            "l2": "flushed between timed steps (256 MiB write) and inputs larger than L2",
            "parallelism": f"replicas x{world}",
        },
        "build_ms": ms_per_step,
        "config1_ms": config1_ms,
        "stage_ms": {name: float(v) for name, v in zip(
            ["emit_bounds", "morton_hist", "sort_4_passes", "karras", "aggregate", "depth_scan", "wide_finish"],
            stage_ms)},
        "roofline": {
            "kernel": "onesweep_pass_kernel",
            "bound": "hbm",
            "achieved": sort_achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": sort_achieved / peak,
            "peak_kind": peak_kind,
            "traffic": None,
            "algorithmic_bytes_per_launch": SORT_PASS_BYTES_PER_PAIR * n,
        },
        "roofline_build": {
            "bound": "hbm",
            "achieved": build_achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": build_achieved / peak,
            "bytes_per_leaf": BUILD_BYTES_PER_LEAF,
        },
        "e2e": {"value": e2e_value, "unit": "Mleaves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 128,
                "ms_per_step": e2e_ms},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, builds, wall = oracle_build_throughput(1 << 20, 10.0, 1)
        line["cpu_baseline"] = {"value": v, "unit": "Mleaves/s", "cores": 1, "kind": "port",
                                "sample": f"{builds} oracle builds of 1048576 records, 1 thread, {wall:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    bvh.close()
    bvh1.close()
    dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["build"], default="build")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--records", type=int, default=N_LEAVES, help="records of the build workload")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_build(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
