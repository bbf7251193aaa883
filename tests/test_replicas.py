"""The multi-GPU form of the benchmark is replicas: every rank solves its own
copy of the batch, there is no collective on the data path, and the job's time
is the slowest replica's.  These tests run the host side of that on CPU with
two gloo ranks (no GPU): the max-over-ranks reduction every rank takes, and the
reference arm, which only rank 0 runs."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # the three reductions of a bench run, in the same order on every rank
        got = [bench.max_over_ranks(v, world, "cpu") for v in values[rank]]
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    values = {0: [61.5, 58.25, 70.0], 1: [59.0, 58.75, 64.5]}
    ctx = tmp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [max(a, b) for a, b in zip(values[0], values[1])]
    assert got[0] == want and got[1] == want


def test_max_over_ranks_one_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5


@pytest.mark.parametrize("rank", [1, 3])
def test_reference_arm_runs_on_rank_zero_only(rank):
    env = dict(os.environ, WORLD_SIZE="4", RANK=str(rank), LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
