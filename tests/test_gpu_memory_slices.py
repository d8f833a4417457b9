"""sliceXor (galois_amd64.go:162-203) and AllocAligned (unsafe.go:19-43) on
the device: XOR over aligned and misaligned ranges of every tail length
against the oracle (galMulSliceXor with c = 1 is sliceXor,
galois_noasm.go:9-67), and shards allocated through rsgpu_alloc_shards:
64-byte aligned, disjoint, usable by Encode, freed with the last shard."""
import ctypes
import gc

import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs
from reedsolomon_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [1, 15, 16, 17, 4096 + 3, (1 << 20) + 5])
@pytest.mark.parametrize("skew", [0, 3])
def test_slice_xor_vs_oracle(size, skew):
    rng = np.random.default_rng(size + skew)
    a = rng.integers(0, 256, size + skew, dtype=np.uint8)
    b = rng.integers(0, 256, size + skew, dtype=np.uint8)
    want = b[skew:].copy()
    O.gal_mul_slice(1, a[skew:].copy(), want, xor=True)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    rs.slice_xor(da[skew:], db[skew:])
    got = db.cpu().numpy()
    assert np.array_equal(got[skew:], want)
    assert np.array_equal(got[:skew], b[:skew])  # bytes before the range untouched


@pytest.mark.parametrize("each", [1, 63, 64, 1000, 1 << 20])
def test_alloc_aligned_shards(each):
    k, p = 10, 4
    enc = rs.New(k, p)
    sh = enc.AllocAligned(each)
    assert len(sh) == k + p
    ptrs = [t.data_ptr() for t in sh]
    assert all(x % 64 == 0 for x in ptrs)
    assert all(b - a >= each for a, b in zip(ptrs, ptrs[1:]))
    rng = np.random.default_rng(each)
    data = [rng.integers(0, 256, each, dtype=np.uint8) for _ in range(k)]
    for i in range(k):
        sh[i].copy_(torch.from_numpy(data[i]))
    enc.Encode(sh)
    want = data + [np.zeros(each, np.uint8) for _ in range(p)]
    O.rs_encode(k, p, want)
    for i in range(k + p):
        assert np.array_equal(sh[i].cpu().numpy(), want[i]), i
    torch.cuda.synchronize()
    del sh
    gc.collect()


def test_alloc_shards_c_abi():
    lib = L.lib()
    ctx = rs.Context.get(0)
    out = (ctypes.c_void_p * 5)()
    assert lib.rsgpu_alloc_shards(ctx.handle, 5, 100, out) == 0
    assert all(out[i] % 64 == 0 for i in range(5))
    assert [out[i + 1] - out[i] for i in range(4)] == [128] * 4
    assert lib.rsgpu_free(ctx.handle, ctypes.c_void_p(out[0])) == 0
    assert lib.rsgpu_alloc_shards(ctx.handle, 0, 100, out) != 0
