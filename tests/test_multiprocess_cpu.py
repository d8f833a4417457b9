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


def test_bench_spawns_its_ranks_without_a_launcher():
    """`bench.py --gpus 2` started without torchrun starts two ranks itself;
    the reference arm prints one line, from rank 0, naming both GPUs' worth
    of ranks and the same config as the product arm."""
    import json
    import subprocess
    env = dict(os.environ)
    for v in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(v, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    sys.path.insert(0, ROOT)
    import bench
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
    assert lines[0]["config"] == bench.workload_config(2)


def test_bench_refuses_a_rank_count_mismatch():
    import subprocess
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and "must match" in r.stderr
