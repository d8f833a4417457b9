"""Split / Join on device buffers against the oracle (reedsolomon.go:1803-1898,
leopard.go:320-370), and the split -> encode -> lose -> reconstruct -> join
workflow of the reference's examples."""
import io

import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu


def new(k, p, leo):
    return rs.New(k, p, rs.WithLeopardGF16()) if leo else rs.New(k, p)


@pytest.mark.parametrize("k,p,leo", [(10, 4, False), (5, 3, False), (17, 3, False), (1, 0, False), (10, 4, True),
                                     (40, 24, True)])
@pytest.mark.parametrize("length", [1, 63, 640, 1000, 4096 + 7, 1 << 20])
def test_split_matches_oracle_and_joins_back(k, p, leo, length):
    rng = np.random.default_rng(length + k)
    data = rng.integers(0, 256, length, dtype=np.uint8)
    rc, want = O.split(k, p, data, leopard=leo)
    assert rc == 0
    enc = new(k, p, leo)
    buf = torch.from_numpy(data).cuda()
    shards = enc.Split(buf)
    assert len(shards) == k + p
    for i in range(k + p):
        assert np.array_equal(shards[i].cpu().numpy(), want[i]), i
    out = torch.zeros(length, dtype=torch.uint8, device="cuda")
    enc.Join(out, shards, length)
    assert np.array_equal(out.cpu().numpy(), data)
    host = io.BytesIO()
    enc.Join(host, shards, length)
    assert host.getvalue() == data.tobytes()


def test_split_uses_spare_capacity():
    k, p, length = 4, 2, 1001
    enc = rs.New(k, p)
    per = (length + k - 1) // k
    buf = torch.full(((k + p) * per + 17,), 0xAB, dtype=torch.uint8, device="cuda")
    data = np.random.default_rng(3).integers(0, 256, length, dtype=np.uint8)
    buf[:length] = torch.from_numpy(data).cuda()
    shards = enc.SplitCap(buf, length, buf.numel())
    base = buf.data_ptr()
    assert all(base <= s.data_ptr() < base + buf.numel() for s in shards)  # no padding allocation
    rc, want = O.split(k, p, data)
    for i in range(k + p):
        assert np.array_equal(shards[i].cpu().numpy(), want[i])   # the spare bytes were zeroed


def test_split_join_errors():
    enc = rs.New(6, 3)
    with pytest.raises(rs.ErrShortData):
        enc.Split(torch.zeros(0, dtype=torch.uint8, device="cuda"))
    shards = enc.Split(torch.arange(600, dtype=torch.int32, device="cuda").to(torch.uint8))
    out = torch.zeros(600, dtype=torch.uint8, device="cuda")
    with pytest.raises(rs.ErrTooFewShards):
        enc.Join(out, shards[:5], 600)
    with pytest.raises(rs.ErrReconstructRequired):
        enc.Join(out, [None] + shards[1:], 600)
    with pytest.raises(rs.ErrShortData):
        enc.Join(out, shards, 601)


@pytest.mark.parametrize("leo", [False, True])
def test_split_encode_reconstruct_join_workflow(leo):
    k, p, length = 10, 4, (3 << 20) + 123
    rng = np.random.default_rng(9)
    data = rng.integers(0, 256, length, dtype=np.uint8)
    enc = new(k, p, leo)
    shards = enc.Split(torch.from_numpy(data).cuda())
    enc.Encode(shards)
    assert enc.Verify(shards)
    lost = [1, 5, 11, 13]
    damaged = [None if i in lost else s for i, s in enumerate(shards)]
    enc.Reconstruct(damaged)
    out = torch.zeros(length, dtype=torch.uint8, device="cuda")
    enc.Join(out, damaged, length)
    assert np.array_equal(out.cpu().numpy(), data)
