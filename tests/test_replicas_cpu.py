"""The multi-process (replica) plumbing of bench.py on the CPU, two gloo ranks.

The path does not shard: under torchrun every rank solves its own systems on
its own GPU and the only collectives are the timing ones (a barrier before a
timed region, the slowest replica's time after it, and, for the serving
stream, every replica's latencies gathered). These tests run those steps
with world size 2 on the gloo backend, and the reference arm as torchrun
would launch it (rank 0 alone measures and prints; the other rank exits 0
without work). No GPU is touched."""

import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import numpy as np
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # each replica's time: the job's is the slowest one's, on every rank
        got = bench.max_over_ranks(dist, 1.0 + 2.5 * rank)
        # the serving arm's gather: every replica's latencies in one list
        parts = [None] * world
        dist.all_gather_object(parts, {"lat": np.full(3, float(rank)), "t0": 10 * rank, "t1": 10 * rank + 7})
        lat = np.concatenate([q["lat"] for q in parts])
        span = max(q["t1"] for q in parts) - min(q["t0"] for q in parts)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got, "lat": lat.tolist(), "span": span}, f)
    finally:
        dist.destroy_process_group()


def test_slowest_replica_sets_the_time_on_every_rank(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        got = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert got["max"] == 3.5
        assert got["lat"] == [0.0, 0.0, 0.0, 1.0, 1.0, 1.0]
        assert got["span"] == 17


def test_one_process_keeps_its_own_time():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, 4.25) == 4.25


def test_reference_arm_with_two_ranks_prints_one_line_from_rank_zero(oracle):
    # the environment torchrun gives each rank (its own argument parser takes
    # a short `--n` after the script for an abbreviation of its options, so
    # the two ranks are started directly)
    world, port = 2, str(_free_port())
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--n", "96", "--steps", "2",
           "--warmup", "1"]
    procs = []
    for r in range(world):
        env = {**os.environ, "OMP_NUM_THREADS": "1", "RANK": str(r), "LOCAL_RANK": str(r),
               "WORLD_SIZE": str(world), "LOCAL_WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
               "MASTER_PORT": port}
        procs.append(subprocess.Popen(cmd, cwd=ROOT, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=300)
            outs.append((p.returncode, out, err))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    for rc, out, err in outs:
        assert rc == 0, err[-2000:]
    assert outs[1][1].strip() == "", "only rank 0 prints"
    lines = [ln for ln in outs[0][1].splitlines() if ln.startswith("{")]
    assert len(lines) == 1, outs[0][1]
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2
    assert line["config"]["parallelism"] == "replicas x2"
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 1


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
