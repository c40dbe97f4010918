"""The benchmark's multi-rank plumbing, run as two gloo ranks on the CPU: the process group comes up
from the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR 127.0.0.1), timings are
the maximum over ranks, the barrier passes on every rank, and under the reference arm only rank 0
works and prints (the other ranks return at once, without output). On the GPU box the same code
runs over NCCL with one process per GPU."""
import json
import multiprocessing as mp
import os
import socket
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir):
    import argparse
    import contextlib
    import io

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import torch.distributed as dist

    import bench

    got_world, got_rank, local = bench.dist_setup()
    res = {"world": got_world, "rank": got_rank, "local": local, "backend": dist.get_backend()}
    res["max"] = bench.max_over_ranks(1.5 * (rank + 1), got_world)
    bench.barrier(got_world)
    args = argparse.Namespace(workload="trace", steps=1, warmup=0, gpus=world, no_cpu_baseline=True)
    if rank != 0:
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            bench.run_reference(args, got_world, got_rank)
        res["reference_output"] = out.getvalue()
    line = bench.base_line(args, got_world, "m", 1.0, "u", 1.0, {"workload": "w"})
    res["n_gpus"] = line["n_gpus"]
    bench.barrier(got_world)
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks(tmp_path):
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0] * world
    results = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, res in enumerate(results):
        assert (res["world"], res["rank"], res["local"]) == (world, r, r)
        assert res["backend"] == "gloo"
        assert res["max"] == 1.5 * world  # every rank sees the slowest rank's time
        assert res["n_gpus"] == world
    assert results[1]["reference_output"] == ""
