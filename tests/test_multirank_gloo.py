"""The N>1 plumbing of bench.py on CPU, with world_size-2 gloo process groups.

The hot path does not shard (replicas only): every rank advances its own
replica, and the only collectives are the barrier and the max-over-ranks of
the timed interval.  These tests run that plumbing without a GPU: the
reduction gives every rank the slowest rank's time, each rank gets its own
replica seed, and the reference arm launched by torchrun on two ranks prints
exactly one JSON line (rank 0) while the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slowest = bench.max_over_ranks(torch, dist, 10.0 + 5.0 * rank, device="cpu")
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"slowest": slowest, "seed": bench.replica_seed(rank)}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [g["slowest"] for g in got] == [15.0, 15.0]
    assert len({g["seed"] for g in got}) == world


def test_max_over_ranks_without_process_group():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, None, 3.25) == 3.25


def test_reference_arm_under_torchrun_prints_one_line():
    sys.path.insert(0, ROOT)
    from oracle.oracle import REF_OMP_LIB
    if not os.path.exists(REF_OMP_LIB):
        pytest.skip("oracle/_ref not built (the reference's C sources were absent at build time)")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
