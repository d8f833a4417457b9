"""Leopard GF(2^16) past one CTA's shared memory (more than 2048 shard
pointers or transform rows, up to the reference's 65536 shards,
leopard.go:51-70): encode and reconstruct run as passes over a work buffer
in HBM and must give the oracle's bytes.  Geometries cover each boundary:
a decode transform past 2048 rows with an encode that still fits one CTA
(1900+148), more shards than one launch's pointer list with m = 1024
(3000+1000), multi-pass transforms (8192+4096), the maximum (32768+32768,
65536-row decode), and many small blocks (5000+3, m = 4)."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu

GEOS = [(1900, 148, 256), (3000, 1000, 128), (8192, 4096, 64), (32768, 32768, 64), (5000, 3, 192)]


def device_shards(arrs):
    size = len(arrs[0])
    pool = torch.from_numpy(np.concatenate(arrs)).cuda()
    return [pool[i * size:(i + 1) * size] for i in range(len(arrs))]


@pytest.mark.parametrize("k,p,size", GEOS)
def test_large_leopard_encode_and_reconstruct(k, p, size):
    rng = np.random.default_rng(k * 7 + p)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(16, k, p, ref) == 0
    enc = rs.New(k, p, rs.WithLeopardGF16())
    sh = device_shards(ref[:k] + [np.zeros(size, np.uint8) for _ in range(p)])
    enc.Encode(sh)
    got = torch.stack(sh[k:]).cpu().numpy()
    for j in range(p):
        assert np.array_equal(got[j], ref[k + j]), j
    assert enc.Verify(sh)
    # erase p shards (data and parity mixed) and rebuild them
    lost = sorted(rng.choice(k + p, size=p, replace=False).tolist())
    present = [0 if i in lost else 1 for i in range(k + p)]
    want = [r.copy() for r in ref]
    for i in lost:
        want[i][:] = 0
    rc, _ = O.leo_reconstruct(16, k, p, want, present)
    assert rc == 0
    for data_only in (False, True):
        work = [None if i in lost else sh[i] for i in range(k + p)]
        (enc.ReconstructData if data_only else enc.Reconstruct)(work)
        for i in lost:
            if data_only and i >= k:
                assert work[i] is None
                continue
            out = work[i].cpu().numpy()
            assert np.array_equal(out, ref[i]), (data_only, i)
            assert np.array_equal(out, want[i]), (data_only, i)


def test_large_leopard_host_buffers():
    """The host-buffer path stages every shard in column chunks and runs the
    same large-geometry transforms per chunk."""
    k, p, size = 3000, 1000, 4096
    rng = np.random.default_rng(11)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(16, k, p, ref) == 0
    enc = rs.New(k, p, rs.WithLeopardGF16())
    ht = [torch.from_numpy(r.copy()) for r in ref[:k]] + [torch.zeros(size, dtype=torch.uint8) for _ in range(p)]
    enc.Encode(ht)
    for j in range(p):
        assert np.array_equal(ht[k + j].numpy(), ref[k + j]), j
    lost = sorted(rng.choice(k + p, size=p, replace=False).tolist())
    work = [None if i in lost else ht[i] for i in range(k + p)]
    enc.Reconstruct(work)
    for i in lost:
        assert np.array_equal(work[i].numpy(), ref[i]), i
