"""The request server: continuous batching, HBM-budget admission, and results
that are identical alone and in a mix (exact GF arithmetic: bit-exact)."""
import threading
import time

import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu

GEOS = [(6, 3, 0), (10, 4, 0), (17, 3, 0), (100, 20, 1)]  # (k, p, leopard); the last is GF(2^16)


def rand_shards(rng, k, p, size):
    data = [torch.from_numpy(rng.integers(0, 256, size, dtype=np.uint8)).cuda() for _ in range(k)]
    return data + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]


def host(ptr, size):
    out = torch.empty(size, dtype=torch.uint8)
    rs.memcpy(out.data_ptr(), ptr, size)
    return out.numpy()


def build_requests(seed, n):
    """Encode requests on fresh stripes and reconstruct requests on encoded
    stripes, each with its expected bytes computed alone through the Encoder API."""
    rng = np.random.default_rng(seed)
    reqs, expect = [], []
    for i in range(n):
        k, p, leo = GEOS[int(rng.integers(0, len(GEOS)))]
        size = int(np.exp(rng.uniform(np.log(4096), np.log(65536)))) // 64 * 64
        enc = rs.New(k, p, rs.WithLeopardGF16()) if leo else rs.New(k, p)
        if rng.random() < 0.6:
            sh = rand_shards(rng, k, p, size)
            alone = [s.clone() for s in sh]
            enc.Encode(alone)
            reqs.append({"op": "encode", "k": k, "p": p, "shards": sh, "leopard": leo, "tag": i})
            expect.append({j: alone[j].cpu().numpy() for j in range(k, k + p)})
        else:
            sh = rand_shards(rng, k, p, size)
            enc.Encode(sh)
            e = int(rng.integers(1, p + 1))
            lost = sorted(int(x) for x in rng.choice(k + p, size=e, replace=False))
            present = [0 if j in lost else 1 for j in range(k + p)]
            alone = [None if j in lost else sh[j] for j in range(k + p)]
            enc.Reconstruct(alone)
            mine = [None if j in lost else sh[j] for j in range(k + p)]
            if rng.random() < 0.5:  # caller-provided output buffers for half of them
                for j in lost:
                    mine[j] = torch.zeros(size, dtype=torch.uint8, device="cuda")
            reqs.append({"op": "reconstruct", "k": k, "p": p, "shards": mine, "present": present,
                         "leopard": leo, "tag": i})
            expect.append({j: alone[j].cpu().numpy() for j in lost})
    return reqs, expect


def check_results(srv, reqs, expect, tickets):
    for r, exp, t in zip(reqs, expect, tickets):
        ptrs = srv.outputs(t)
        size = max(len(s) for s in r["shards"] if s is not None)
        for j, want in exp.items():
            assert ptrs[j], (r["tag"], j)
            assert np.array_equal(host(ptrs[j], size), want), (r["op"], r["k"], r["p"], j)


def test_server_results_alone_equal_mix():
    reqs, expect = build_requests(7, 120)
    srv = rs.Server(arena_bytes=256 << 20, inflight_budget=512 << 20, max_batch=32, streams=4)
    rng = np.random.default_rng(8)
    arrivals = np.cumsum(rng.exponential(50.0, len(reqs)))  # Poisson, 20k req/s offered
    tickets = srv.replay(reqs, arrivals)
    srv.wait_idle(60000)
    done = srv.poll_detailed()
    assert len(done) == len(reqs) and all(st == 0 for _, _, st, _, _ in done)
    assert all(0 <= q <= lat for _, _, _, lat, q in done)  # admission wait is part of the latency
    check_results(srv, reqs, expect, tickets)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
    for t in tickets:
        srv.release(t)
    srv.close()


def test_server_hbm_admission_waits_for_release():
    """An arena that holds two requests' outputs: later requests wait until
    earlier outputs are released, and the in-flight budget is respected."""
    k, p, size = 10, 4, 1 << 20
    rng = np.random.default_rng(3)
    sh = rand_shards(rng, k, p, size)
    enc = rs.New(k, p)
    enc.Encode(sh)
    present = [0, 0, 0, 0] + [1] * 10  # 4 data outputs of 1 MiB each per request
    srv = rs.Server(arena_bytes=2 * 4 * size, inflight_budget=32 * size, max_batch=8, streams=2)
    tickets = [srv.submit("reconstruct", k, p, [None] * 4 + sh[4:], present) for _ in range(6)]
    finished, released = set(), 0
    deadline = time.time() + 30
    while len(finished) < 6 and time.time() < deadline:
        for t, _, st, _ in srv.poll():
            assert st == 0
            finished.add(t)
            for j, ptr in enumerate(srv.outputs(t)[:4]):
                assert np.array_equal(host(ptr, size), sh[j].cpu().numpy())
            srv.release(t)
            released += 1
        time.sleep(0.001)
    assert len(finished) == 6 and released == 6
    assert srv.stats()["max_inflight_bytes"] <= 32 * size
    srv.close()


def test_server_verify_errors_and_timeouts():
    rng = np.random.default_rng(5)
    k, p, size = 6, 3, 1 << 16
    sh = rand_shards(rng, k, p, size)
    rs.New(k, p).Encode(sh)
    srv = rs.Server(arena_bytes=1 << 20, inflight_budget=1 << 30, max_batch=16, streams=2)
    t_ok = srv.submit("verify", k, p, sh)
    bad = [s.clone() for s in sh]
    bad[k][7] ^= 1
    t_bad = srv.submit("verify", k, p, bad)
    t_err = srv.submit("reconstruct", k, p, [None] * (p + 1) + sh[p + 1:], [0] * (p + 1) + [1] * (k - 1))
    srv.wait_idle(30000)
    got = {t: st for t, _, st, _ in srv.poll()}
    assert got[t_ok] == 0 and got[t_bad] == 0 and got[t_err] == rs.ErrTooFewShards.code
    assert srv.verify_result(t_ok) and not srv.verify_result(t_bad)
    # a large request: waiting 0 ms while it runs times out cleanly, then completes
    big = rand_shards(rng, 10, 4, 64 << 20)
    srv.submit("encode", 10, 4, big)
    with pytest.raises(rs.ErrTimeout):
        srv.wait_idle(0)
    srv.wait_idle(30000)
    srv.close()


def test_server_stuck_producer_leaves_server_idle():
    """A producer that stops submitting: the server drains what it got and idles;
    shutting it down does not wait on the producer."""
    rng = np.random.default_rng(9)
    srv = rs.Server(arena_bytes=1 << 20, inflight_budget=1 << 30, max_batch=16, streams=2)
    sh = [rand_shards(rng, 6, 3, 4096) for _ in range(5)]
    stop_after = 3

    def producer():
        for i in range(stop_after):  # then stops feeding for good
            srv.submit("encode", 6, 3, sh[i])

    th = threading.Thread(target=producer)
    th.start()
    th.join(10)
    srv.wait_idle(10000)
    assert len(srv.poll()) == stop_after
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 10
