"""The multi-rank (replicas) path of bench.py on CPU: two gloo ranks.

A matrix does not shard across GPUs for these workloads, so `bench.py --gpus N`
runs N independent replicas; the only cross-rank steps are the barriers around
the timed region, the max of the per-rank times and the whole-job total.  These
are exercised here with the gloo backend (world size 2, 127.0.0.1), as the
NCCL run does them on a GPU node.
"""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # each replica reports its own time; the job's time is the slowest one
        ms = [12.5, 20.0][rank]
        ms_max = bench.max_over_ranks(ms, world)
        value = bench.replica_throughput(world, 846e6, 10, ms_max)
        bench.barrier(world)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{ms_max} {value}\n")
    finally:
        dist.destroy_process_group()


def test_replicas_max_time_and_total(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        ms_max, value = map(float, open(tmp_path / f"rank{r}.txt").read().split())
        assert ms_max == 20.0  # every rank sees the slowest rank's time
        # two replicas of 10 applications of 846 MB in 20 ms: 846 GB/s in total
        assert value == pytest.approx(2 * 846e6 * 10 / 0.020 / 1e9)


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the CPU reference; the others exit 0 at once."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
