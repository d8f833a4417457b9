"""Seeded random sweep over geometries, sizes and erasure sets, bit-exact
against the oracle: Leopard GF(2^16) up to 2048 shards (every block size m
from 1 to 1024, compact and full staged tables) and past one CTA, Leopard
GF(2^8) with ceilPow2(p) + k <= 256, and classic codes of up to 47 + 19
shards with ragged sizes and every GF(2^8) kernel variant forced in turn
(Encode, Verify, Reconstruct of a random erasure set).  The reference's
tests draw random shards the same way (reedsolomon_test.go:306-418,
leopard_test.go:12-124)."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu


def dev_pool(arrs):
    size = len(arrs[0])
    pool = torch.from_numpy(np.concatenate(arrs)).cuda()
    return [pool[i * size:(i + 1) * size] for i in range(len(arrs))]


def run_leopard(rng, gf, total_max, cases, max_chunks):
    done = 0
    for _ in range(cases):
        p = int(rng.integers(1, min(600, total_max // 2) + 1))
        k = int(rng.integers(1, total_max - p + 1))
        m = 1 << (p - 1).bit_length()
        if gf == 8 and m + k > 256:
            continue
        if gf == 16 and ((k + m - 1) // m - 1) * m + 2 * m - 2 >= 65535:
            continue
        size = 64 * int(rng.integers(1, max_chunks + 1))
        ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
              [np.zeros(size, np.uint8) for _ in range(p)]
        assert O.leo_encode(gf, k, p, ref) == 0
        enc = rs.New(k, p, rs.WithLeopardGF16() if gf == 16 else rs.WithLeopardGF())
        sh = dev_pool(ref[:k] + [np.zeros(size, np.uint8)] * p)
        enc.Encode(sh)
        for j in range(p):
            assert np.array_equal(sh[k + j].cpu().numpy(), ref[k + j]), (gf, k, p, size, j)
        lost = sorted(rng.choice(k + p, size=int(rng.integers(1, p + 1)), replace=False).tolist())
        work = [None if i in lost else sh[i] for i in range(k + p)]
        enc.Reconstruct(work)
        for i in lost:
            assert np.array_equal(work[i].cpu().numpy(), ref[i]), (gf, k, p, size, lost, i)
        done += 1
    return done


def test_leopard16_random_geometries():
    assert run_leopard(np.random.default_rng(2101), 16, 2048, 120, 4) >= 100


def test_leopard16_random_geometries_past_one_cta():
    assert run_leopard(np.random.default_rng(2102), 16, 6000, 6, 2) >= 5


def test_leopard8_random_geometries():
    assert run_leopard(np.random.default_rng(2103), 8, 256, 120, 8) >= 90


def test_classic_random_geometries_every_variant():
    rng = np.random.default_rng(2104)
    lib = rs.lib()
    nv = lib.rsgpu_num_variants()
    try:
        for c in range(120):
            k, p = int(rng.integers(1, 48)), int(rng.integers(1, 20))
            size = int(rng.integers(1, 70000))
            ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
                  [np.zeros(size, np.uint8) for _ in range(p)]
            O.rs_encode(k, p, ref)
            v = c % (nv + 1) - 1  # -1: the default choice
            assert lib.rsgpu_force_variant(v) == 0
            enc = rs.New(k, p)
            sh = dev_pool(ref[:k] + [np.zeros(size, np.uint8)] * p)
            enc.Encode(sh)
            for j in range(p):
                assert np.array_equal(sh[k + j].cpu().numpy(), ref[k + j]), (k, p, size, v, j)
            assert enc.Verify(sh), (k, p, size, v)
            lost = sorted(rng.choice(k + p, size=int(rng.integers(1, p + 1)), replace=False).tolist())
            work = [None if i in lost else sh[i] for i in range(k + p)]
            enc.Reconstruct(work)
            for i in lost:
                assert np.array_equal(work[i].cpu().numpy(), ref[i]), (k, p, size, v, lost, i)
    finally:
        lib.rsgpu_force_variant(-1)
