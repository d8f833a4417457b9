"""The N > 1 bench plumbing on CPU: two gloo ranks over 127.0.0.1.

bench.py runs one process per GPU; each encodes its own stripe (weak
scaling) and the timed region is reduced to the slowest rank.  These tests
exercise that host logic without a GPU: the max-over-ranks reduction, the
per-rank stripe seeds, and the reference arm's rank-0-only output.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(1.5 + rank, world, "cpu")
        w, r, local = bench.dist_setup(None)
        out.put((rank, ms, bench.stripe_seed(r), w, local))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_stripe_partition_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[1] for g in got] == [2.5, 2.5]           # every rank sees the slowest rank's time
    assert len({g[2] for g in got}) == world           # independent stripes per rank
    assert all(g[3] == world for g in got) and [g[4] for g in got] == [0, 1]


def test_reference_arm_prints_on_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.main() == 0
    assert buf.getvalue() == ""


def test_single_rank_max_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25
