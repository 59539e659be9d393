"""The bench's multi-process plumbing on CPU (gloo, two ranks): replicas'
device times reduce to the slowest rank's, and the reference arm runs and
prints on rank 0 only (the other ranks exit 0 without work)."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ranks(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_dist(world, "gloo")
    vals = bench.max_over_ranks([10.0 * (rank + 1), 5.0 - rank], world, device="cpu")
    out[rank] = vals
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world, port = 2, 29517
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_ranks, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1] == [20.0, 5.0]


def test_single_rank_times_pass_through():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_other_ranks_exit_without_work(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
               MASTER_PORT="29518")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
