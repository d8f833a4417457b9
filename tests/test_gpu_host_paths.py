"""GPU parity of the host-buffer entry points (PCIe copies inside the call)
against the oracle: Verify, EncodeIdx, Update, DecodeIdx and ReconstructSome
on host shards (pinned and pageable), classic and Leopard, called through the
Python mirror (which routes host tensors to the *_host C-ABI functions) and
directly through ctypes.  Sizes cross several pipeline chunks (1 MiB each)
and end on a ragged tail."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs
from reedsolomon_b200 import _lib as L

pytestmark = pytest.mark.gpu


def hostt(a, pinned=False):
    t = torch.from_numpy(np.ascontiguousarray(a).copy())
    return t.pin_memory() if pinned else t


def encoded(rng, k, p, size):
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.rs_encode(k, p, sh) == 0
    return sh


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("k,p,size", [(10, 4, (3 << 20) + 7), (6, 3, 1000), (20, 10, 65536)])
def test_verify_host_classic(k, p, size, pinned):
    rng = np.random.default_rng(k + size)
    ref = encoded(rng, k, p, size)
    enc = rs.New(k, p)
    sh = [hostt(a, pinned) for a in ref]
    assert enc.Verify(sh)
    for pos in (0, size // 2, size - 1):
        sh[k + p - 1][pos] ^= 1
        assert not enc.Verify(sh)
        sh[k + p - 1][pos] ^= 1
    assert enc.Verify(sh)
    ok = ctypes.c_int(-1)
    assert L.lib().rsgpu_verify_host(enc._h, L.ptr_array([t.data_ptr() for t in sh]), size, ctypes.byref(ok)) == 0
    assert ok.value == 1


@pytest.mark.parametrize("gf,k,p,size", [(16, 300, 60, 8192), (8, 100, 28, 64 * 1024 + 64)])
def test_verify_host_leopard(gf, k, p, size):
    rng = np.random.default_rng(gf)
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(gf, k, p, sh) == 0
    enc = rs.New(k, p, rs.WithLeopardGF16() if gf == 16 else rs.WithLeopardGF())
    ht = [hostt(a) for a in sh]
    assert enc.Verify(ht)
    ht[k][size - 1] ^= 0x80
    assert not enc.Verify(ht)


@pytest.mark.parametrize("k,p,size,idx", [(10, 4, (2 << 20) + 100, 3), (5, 3, 777, 0), (17, 3, 65536, 16)])
def test_encode_idx_host(k, p, size, idx):
    rng = np.random.default_rng(size + idx)
    data = rng.integers(0, 256, size, dtype=np.uint8)
    par = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(p)]
    want = [x.copy() for x in par]
    assert O.rs_encode_idx(k, p, data, idx, want) == 0
    ht = [hostt(x) for x in par]
    rs.New(k, p).EncodeIdx(hostt(data), idx, ht)
    for o in range(p):
        assert np.array_equal(ht[o].numpy(), want[o]), o


@pytest.mark.parametrize("k,p,size,changed", [(10, 4, (2 << 20) + 9, (1, 7)), (6, 3, 1000, (0,)),
                                              (40, 8, 2048, tuple(range(0, 40, 3)))])
def test_update_host(k, p, size, changed):
    rng = np.random.default_rng(k * 100 + p)
    ref = encoded(rng, k, p, size)
    new = [None] * k
    for c in changed:
        new[c] = rng.integers(0, 256, size, dtype=np.uint8)
    want = [a.copy() for a in ref]
    assert O.rs_update(k, p, want, new, size) == 0
    sh = [hostt(a) for a in ref]
    rs.New(k, p).Update(sh, [None if x is None else hostt(x) for x in new])
    for i in range(k + p):
        assert np.array_equal(sh[i].numpy(), want[i]), i


@pytest.mark.parametrize("k,p,size", [(10, 4, (2 << 20) + 64), (6, 3, 1000), (17, 3, 65536 + 48)])
def test_decode_idx_host_progressive(k, p, size):
    rng = np.random.default_rng(k + p + size)
    ref = encoded(rng, k, p, size)
    n = k + p
    lost = set(int(x) for x in rng.choice(n, size=p, replace=False))
    expect = [0 if i in lost else 1 for i in range(n)]
    avail = [i for i in range(n) if expect[i]]
    half = (avail[: len(avail) // 2], avail[len(avail) // 2:])
    want = [np.zeros(size, np.uint8) if i in lost else None for i in range(n)]
    for part in half:
        inp = [ref[i] if i in part else None for i in range(n)]
        assert O.rs_decode_idx(k, p, want, expect, inp, size) == 0
    dst = [hostt(np.zeros(size, np.uint8)) if i in lost else None for i in range(n)]
    enc = rs.New(k, p)
    for part in half:
        enc.DecodeIdx(dst, expect, [hostt(ref[i]) if i in part else None for i in range(n)])
    for i in lost:
        assert np.array_equal(dst[i].numpy(), want[i]), i
        assert np.array_equal(dst[i].numpy(), ref[i]), i
    # merging mode: dst ^= input
    a = [hostt(ref[0]), None] + [None] * (n - 2)
    b = [hostt(ref[1]), None] + [None] * (n - 2)
    enc.DecodeIdx(a, None, b)
    assert np.array_equal(a[0].numpy(), ref[0] ^ ref[1])


@pytest.mark.parametrize("kind", ["data_only", "all"])
def test_reconstruct_some_host_classic(kind):
    k, p, size = 10, 4, (2 << 20) + 48
    rng = np.random.default_rng(7)
    ref = encoded(rng, k, p, size)
    lost = [1, 4, 11, 13]
    required = [i in (1, 11) for i in range(k + p)] if kind == "all" else [i == 4 for i in range(k)]
    sh = [None if i in lost else hostt(ref[i]) for i in range(k + p)]
    rs.New(k, p).ReconstructSome(sh, required)
    for i in range(len(required)):
        if required[i]:
            assert sh[i] is not None and np.array_equal(sh[i].numpy(), ref[i]), i
    for i in lost:
        if not (i < len(required) and required[i]):
            assert sh[i] is None, i


def test_reconstruct_some_host_leopard():
    k, p, size, gf = 200, 40, 4096, 16
    rng = np.random.default_rng(3)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(gf, k, p, ref) == 0
    enc = rs.New(k, p, rs.WithLeopardGF16())
    lost = sorted(rng.choice(k + p, size=p, replace=False).tolist())
    for required in ([True] * (k + p), [False] * k):  # full length: parity too; data length: data only
        sh = [None if i in lost else hostt(ref[i]) for i in range(k + p)]
        enc.ReconstructSome(sh, required)
        for i in lost:
            if i < k or len(required) == k + p:
                assert sh[i] is not None and np.array_equal(sh[i].numpy(), ref[i]), i
            else:
                assert sh[i] is None


def test_host_entry_points_refuse_mixed_and_leopard_progressive():
    k, p, size = 6, 3, 256
    rng = np.random.default_rng(9)
    ref = encoded(rng, k, p, size)
    enc = rs.New(k, p)
    mixed = [hostt(a) for a in ref]
    mixed[0] = mixed[0].cuda()
    with pytest.raises(rs.ErrNotSupported):
        enc.Verify(mixed)
    lib = L.lib()
    leo = rs.New(k, p, rs.WithLeopardGF16())
    pa = L.ptr_array([hostt(a).data_ptr() for a in ref[k:]])
    assert lib.rsgpu_encode_idx_host(leo._h, hostt(ref[0]).data_ptr(), 0, pa, size) == -7


@pytest.mark.parametrize("layout", ["block_pinned", "block_pageable", "separate_pinned"])
@pytest.mark.parametrize("k,p,size", [(10, 4, (9 << 20) + 48), (4, 2, 1000)])
def test_encode_and_reconstruct_host_layouts(layout, k, p, size):
    """Host shards that are consecutive pieces of one block (one 2D copy per
    pipeline chunk and direction) or separate allocations (per-row copies,
    or a rejected 2D copy falling back to them), with full chunks, the
    halving tail chunks and a ragged end: the parity and rebuilt shards
    equal the oracle's."""
    rng = np.random.default_rng(size + k)
    ref = encoded(rng, k, p, size)
    if layout.startswith("block"):
        block = torch.zeros((k + p) * size, dtype=torch.uint8)
        if layout == "block_pinned":
            block = block.pin_memory()
        sh = [block[i * size:(i + 1) * size] for i in range(k + p)]
    else:
        sh = [torch.zeros(size, dtype=torch.uint8).pin_memory() for _ in range(k + p)]
    for i in range(k):
        sh[i].copy_(torch.from_numpy(ref[i]))
    enc = rs.New(k, p)
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(sh[i].numpy(), ref[i]), (layout, i)
    # lost data shards 0..p-1: the survivors the decode reads are the
    # consecutive rows p..k+p-1, one run (the rebuilt shards are new tensors);
    # then scattered erasures: several runs of survivors
    for lost in (list(range(p)), sorted(rng.choice(k + p, size=p, replace=False).tolist())):
        work = [None if i in lost else sh[i] for i in range(k + p)]
        enc.Reconstruct(work)
        for i in lost:
            assert np.array_equal(work[i].numpy(), ref[i]), (layout, lost, i)


@pytest.mark.parametrize("leopard", [True, False])
def test_host_chunks_stay_aligned_with_mixed_layouts(leopard):
    """Host shards in runs of different lengths (data shards 0-1 in one block,
    2 alone, the parity in another block: 1.5 rows per 2D copy) make the
    pipeline's minimum chunk 1 MiB / 1.5, which must still be rounded to the
    codec's alignment (64 bytes for Leopard) for every chunk but the last."""
    k, p, size = 3, 2, 3 << 20
    rng = np.random.default_rng(99 + leopard)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    if leopard:
        assert O.leo_encode(16, k, p, ref) == 0
        enc = rs.New(k, p, rs.WithLeopardGF16())
    else:
        assert O.rs_encode(k, p, ref) == 0
        enc = rs.New(k, p)
    data01 = torch.from_numpy(np.concatenate(ref[:2])).pin_memory()
    data2 = torch.from_numpy(ref[2].copy()).pin_memory()
    par = torch.zeros(p * size, dtype=torch.uint8).pin_memory()
    sh = [data01[:size], data01[size:], data2] + [par[j * size:(j + 1) * size] for j in range(p)]
    enc.Encode(sh)
    for j in range(p):
        assert np.array_equal(sh[k + j].numpy(), ref[k + j]), (leopard, j)
