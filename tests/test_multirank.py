"""The multi-rank plumbing of bench.py on CPU: world_size 2 over gloo
(127.0.0.1).  A single scenario does not shard, so N ranks run N replicas;
the only exchange is the max over ranks of the timed region, which every
rank must take at the same point.  The reference arm runs on rank 0 alone."""
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


def _worker(rank, world, port, values, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(values[rank], world, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    values = [1.25, 7.5]
    mp.start_processes(_worker, args=(2, port, values, out), nprocs=2, join=True,
                       start_method="spawn")
    assert dict(out) == {0: 7.5, 1: 7.5}


def test_max_over_ranks_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


@pytest.mark.parametrize("rank", ["1"])
def test_reference_arm_only_rank_zero_prints(rank, tmp_path):
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
