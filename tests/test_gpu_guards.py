"""Out-of-bounds write checks without a sanitizer: every shard sits in one
device allocation between 64-byte canary regions, and every write path
(encode, reconstruct, update, decode_idx, code_some_shards, the batch
kernel, Leopard encode / decode, split) must leave all canaries intact and
produce the oracle's bytes, over odd and tiny shard sizes and misaligned
starts."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu

GUARD = 64
CANARY = 0xA5


class Guarded:
    """n shards of `size` bytes, each preceded and followed by canary bytes;
    `skew` shifts every shard start off the 16-byte grid."""

    def __init__(self, n, size, skew=0):
        self.n, self.size, self.skew = n, size, skew
        self.pitch = GUARD + skew + size + GUARD
        self.buf = torch.full((n * self.pitch,), CANARY, dtype=torch.uint8, device="cuda")
        self.shards = [self.view(i) for i in range(n)]

    def view(self, i):
        start = i * self.pitch + GUARD + self.skew
        return self.buf[start:start + self.size]

    def canaries_intact(self):
        h = self.buf.cpu().numpy().reshape(self.n, self.pitch)
        lead = h[:, :GUARD + self.skew]
        tail = h[:, GUARD + self.skew + self.size:]
        return bool((lead == CANARY).all() and (tail == CANARY).all())


def fill(g, rng, idx):
    for i in idx:
        g.shards[i].copy_(torch.from_numpy(rng.integers(0, 256, g.size, dtype=np.uint8)))


SIZES = [1, 7, 15, 16, 17, 63, 64, 65, 255, 4097, 65536 + 13]


@pytest.mark.parametrize("size", SIZES)
@pytest.mark.parametrize("skew", [0, 1, 8])
def test_classic_paths_stay_in_bounds(size, skew):
    k, p = 10, 4
    rng = np.random.default_rng(size * 3 + skew)
    g = Guarded(k + p, size, skew)
    fill(g, rng, range(k))
    enc = rs.New(k, p)
    enc.Encode(g.shards)
    ref = [s.cpu().numpy().copy() for s in g.shards]
    want = [a.copy() for a in ref]
    for i in range(k, k + p):
        want[i][:] = 0
    O.rs_encode(k, p, want)
    assert all(np.array_equal(ref[i], want[i]) for i in range(k, k + p))
    assert enc.Verify(g.shards)
    lost = [1, 5, 11, 13]
    for i in lost:
        g.shards[i].fill_(0)
    enc.Reconstruct([None if i in lost else s for i, s in enumerate(g.shards)])  # outputs allocated
    cp = list(g.shards)
    present = [0 if i in lost else 1 for i in range(k + p)]
    lib = rs.lib()
    pres = rs._lib.u8_array(present)
    ptrs = rs._lib.ptr_array([s.data_ptr() for s in cp])
    rs.encoder.check(lib.rsgpu_reconstruct(enc._h, ptrs, pres, size, None))  # in place, guarded
    for i in range(k + p):
        assert np.array_equal(g.shards[i].cpu().numpy(), ref[i]), i
    new = [None] * k
    new[3] = torch.from_numpy(rng.integers(0, 256, size, dtype=np.uint8)).cuda()
    enc.Update(g.shards, new)
    assert g.canaries_intact()


@pytest.mark.parametrize("size", [64, 128, 4096, 65536 + 64])
@pytest.mark.parametrize("gf", [16, 8])
def test_leopard_paths_stay_in_bounds(size, gf):
    k, p = (40, 20) if gf == 16 else (30, 10)
    rng = np.random.default_rng(size + gf)
    g = Guarded(k + p, size, 0)
    fill(g, rng, range(k))
    enc = rs.New(k, p, rs.WithLeopardGF16() if gf == 16 else rs.WithLeopardGF())
    enc.Encode(g.shards)
    ref = [s.cpu().numpy().copy() for s in g.shards]
    want = [a.copy() for a in ref]
    for i in range(k, k + p):
        want[i][:] = 0
    O.leo_encode(gf, k, p, want)
    assert all(np.array_equal(ref[i], want[i]) for i in range(k, k + p))
    lost = sorted(int(x) for x in rng.choice(k + p, size=p, replace=False))
    for i in lost:
        g.shards[i].fill_(0)
    lib = rs.lib()
    pres = rs._lib.u8_array([0 if i in lost else 1 for i in range(k + p)])
    ptrs = rs._lib.ptr_array([s.data_ptr() for s in g.shards])
    rs.encoder.check(lib.rsgpu_reconstruct(enc._h, ptrs, pres, size, None))
    for i in range(k + p):
        assert np.array_equal(g.shards[i].cpu().numpy(), ref[i]), i
    assert g.canaries_intact()


def test_batch_kernel_stays_in_bounds():
    rng = np.random.default_rng(5)
    guards, b = [], rs.Batch()
    for size in (1, 17, 64, 1000, 4096, 20000 + 3):
        for skew in (0, 4):
            k, p = int(rng.integers(2, 12)), int(rng.integers(1, 8))
            g = Guarded(k + p, size, skew)
            fill(g, rng, range(k))
            b.add_encode(k, p, g.shards)
            guards.append((k, p, g))
    b.run("persistent")
    for k, p, g in guards:
        ref = [s.cpu().numpy() for s in g.shards]
        want = [a.copy() for a in ref]
        for i in range(k, k + p):
            want[i][:] = 0
        O.rs_encode(k, p, want)
        assert all(np.array_equal(ref[i], want[i]) for i in range(k, k + p))
        assert g.canaries_intact()


def test_split_and_decode_idx_stay_in_bounds():
    k, p, length = 6, 3, 1001
    rng = np.random.default_rng(6)
    enc = rs.New(k, p)
    per = (length + k - 1) // k
    g = Guarded(1, k * per + 5, 0)   # capacity past the data, canaries beyond it
    data = rng.integers(0, 256, length, dtype=np.uint8)
    g.shards[0][:length] = torch.from_numpy(data).cuda()
    shards = enc.SplitCap(g.shards[0], length, g.shards[0].numel())
    enc.Encode(shards)
    assert g.canaries_intact()
    d = Guarded(k + p, per, 3)
    for t in d.shards:
        t.zero_()
    expect = [1] * k + [0] * p
    dst = [None] * k + d.shards[k:]
    enc.DecodeIdx(dst, expect, list(shards[:k]) + [None] * p)
    for i in range(k, k + p):
        assert torch.equal(d.shards[i], shards[i])
    assert d.canaries_intact()
