"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the
timing reduction every rank takes part in, and the reference arm, which
runs on rank 0 only (the other ranks exit 0 without work)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(10.0 + 5.0 * rank, dist)   # rank 1 is the slow one
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_max_over_ranks_gloo():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 15.0, 1: 15.0}


def test_max_over_ranks_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


@pytest.mark.parametrize("rank", [1, 3])
def test_reference_arm_other_ranks_exit_clean(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="4", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "4"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
