"""The N > 1 path of bench.py on CPU: two `gloo` ranks (replicas only: the
path has no exchange step, so the only collectives are the barrier and the
max-over-ranks reduction of the measured times), and the reference arm's rule
that only rank 0 works under torchrun."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        # each replica measured a different time; every rank reports the slowest
        got = bench.max_over_ranks(10.0 + 5.0 * rank, torch.device("cpu"), world)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None, 1) == 3.5


@pytest.mark.parametrize("rank", ["1"])
def test_reference_arm_nonzero_rank_exits_without_work(rank):
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"], env=env,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == ""
