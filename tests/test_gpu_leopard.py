"""GPU parity tests of the Leopard GF(2^16) / GF(2^8) codec against the CPU oracle.

Encode parity and reconstructed bytes are compared bit-exactly with the
oracle's restatement of leopard.go / leopard8.go; round trips must also give
back the original data and the encoder's own parity.
"""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def new(gf, k, p):
    return rs.New(k, p, rs.WithLeopardGF16() if gf == 16 else rs.WithLeopardGF())


# GF(2^16) block sizes m = 1 .. 512: the encode's staged tables are compact
# (no nibble tables for slots = 3 mod 4) for m = 2^even and full for
# m = 2^odd, whose FFT has a distance-2 pass (m = 8, 32, 128, 512 here)
CASES = [(16, 1, 1, 64), (16, 3, 2, 128), (16, 5, 3, 192), (16, 20, 13, 256), (16, 64, 64, 128),
         (16, 300, 60, 128), (16, 500, 300, 64), (16, 10, 4, 4096), (16, 30, 7, 192), (16, 200, 100, 128),
         (16, 100, 16, 64), (16, 70, 20, 128),
         (8, 1, 1, 64), (8, 5, 3, 128), (8, 40, 24, 256), (8, 100, 28, 64), (8, 192, 56, 128)]


@pytest.mark.parametrize("gf,k,p,size", CASES)
def test_encode_matches_oracle(gf, k, p, size):
    rng = np.random.default_rng(gf * 1000 + k * 7 + p)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    sh = [dev(a) for a in ref]
    assert O.leo_encode(gf, k, p, ref) == 0
    enc = new(gf, k, p)
    assert enc.codec == (1 if gf == 16 else 2)
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), ref[i]), (gf, k, p, i)
    assert enc.Verify(sh)
    sh[k][size - 1] ^= 1
    assert not enc.Verify(sh)


@pytest.mark.parametrize("gf,k,p,size", CASES)
def test_reconstruct_matches_oracle(gf, k, p, size):
    rng = np.random.default_rng(gf * 77 + k + p)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    O.leo_encode(gf, k, p, ref)
    enc = new(gf, k, p)
    for trial in range(3):
        e = int(rng.integers(1, p + 1))
        lost = sorted(int(x) for x in rng.choice(k + p, size=e, replace=False))
        present = [0 if i in lost else 1 for i in range(k + p)]
        # oracle on copies with lost shards zeroed
        want = [a.copy() for a in ref]
        for i in lost:
            want[i][:] = 0
        rc, written = O.leo_reconstruct(gf, k, p, want, present, recover_all=True)
        assert rc == 0
        sh = [None if i in lost else dev(ref[i]) for i in range(k + p)]
        enc.Reconstruct(sh)
        for i in lost:
            got = host(sh[i])
            assert np.array_equal(got, want[i]), (gf, k, p, i, "oracle")
            assert np.array_equal(got, ref[i]), (gf, k, p, i, "original")
        # data only
        sh = [None if i in lost else dev(ref[i]) for i in range(k + p)]
        enc.ReconstructData(sh)
        for i in lost:
            if i < k:
                assert np.array_equal(host(sh[i]), ref[i])
            else:
                assert sh[i] is None


def test_leopard16_1000_200_64kib():
    """Leopard GF(2^16) 1000+200 x 64 KiB: encode vs oracle, 200 random erasures, reconstruct."""
    k, p, size = 1000, 200, 65536
    rng = np.random.default_rng(1200)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    sh = [dev(a) for a in ref]
    assert O.leo_encode(16, k, p, ref) == 0
    enc = rs.New(k, p)  # > 256 shards routes to GF(2^16)
    assert enc.codec == 1
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i
    assert enc.Verify(sh)
    lost = sorted(int(x) for x in rng.choice(k + p, size=p, replace=False))
    cp = [None if i in lost else sh[i] for i in range(k + p)]
    enc.Reconstruct(cp)
    for i in lost:
        assert np.array_equal(host(cp[i]), ref[i]), i


def test_leopard8_192_56_256kib():
    """Leopard GF(2^8) 192+56 x 256 KiB with 56 erasures (200+56 indexes past the reference's tables)."""
    k, p, size = 192, 56, 262144
    rng = np.random.default_rng(256)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    sh = [dev(a) for a in ref]
    assert O.leo_encode(8, k, p, ref) == 0
    enc = rs.New(k, p, rs.WithLeopardGF())
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i
    lost = sorted(int(x) for x in rng.choice(k + p, size=p, replace=False))
    cp = [None if i in lost else sh[i] for i in range(k + p)]
    enc.Reconstruct(cp)
    for i in lost:
        assert np.array_equal(host(cp[i]), ref[i]), i
    with pytest.raises(rs.ErrMaxShardNum):
        rs.New(200, 56, rs.WithLeopardGF())


def test_leopard_errors_and_host_path():
    enc = rs.New(10, 4, rs.WithLeopardGF16())
    sh = [torch.zeros(100, dtype=torch.uint8, device="cuda") for _ in range(14)]
    with pytest.raises(rs.ErrInvalidShardSize):
        enc.Encode(sh)
    with pytest.raises(rs.ErrNotSupported):
        enc.EncodeIdx(sh[0][:64], 0, [s[:64] for s in sh[10:]])
    size = 1 << 16
    rng = np.random.default_rng(3)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(10)] + [np.zeros(size, np.uint8) for _ in range(4)]
    O.leo_encode(16, 10, 4, ref)
    hs = [torch.from_numpy(a.copy()).pin_memory() for a in ref[:10]] + \
         [torch.zeros(size, dtype=torch.uint8).pin_memory() for _ in range(4)]
    enc.Encode(hs)
    for i in range(10, 14):
        assert np.array_equal(hs[i].numpy(), ref[i])
    for i in (0, 11, 13):
        hs[i] = None
    enc.Reconstruct(hs)
    for i in (0, 11, 13):
        assert np.array_equal(hs[i].numpy(), ref[i])
    cp = [None, None, None, None, None] + [dev(a) for a in ref[5:]]
    with pytest.raises(rs.ErrTooFewShards):
        rs.New(10, 4, rs.WithLeopardGF16()).Reconstruct(cp)


@pytest.mark.parametrize("gf", [16, 8])
def test_leopard_rejects_misaligned_shards(gf):
    """Shard buffers off a 16-byte boundary are refused on the host before any launch."""
    k, p, size = 5, 3, 128
    base = torch.zeros((k + p) * (size + 16) + 16, dtype=torch.uint8, device="cuda")
    sh = [base[1 + i * (size + 16):1 + i * (size + 16) + size] for i in range(k + p)]
    enc = new(gf, k, p)
    with pytest.raises(rs.ErrNotSupported):
        enc.Encode(sh)
    sh[0] = None
    with pytest.raises(rs.ErrNotSupported):
        enc.Reconstruct(sh)


@pytest.mark.parametrize("gf", [16, 8])
def test_leopard_shards_past_2gib_offsets(gf):
    """Shards longer than 2^31 bytes: Leopard is local to each 64-byte chunk,
    so 64-byte aligned windows across the 32-bit boundary must equal the
    oracle's encode of the same windows, and reconstruct must restore them."""
    k, p = 4, 2
    size = (1 << 31) + 128
    g = torch.Generator(device="cuda").manual_seed(gf)
    sh = [torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g) for _ in range(k)]
    sh += [torch.empty(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    enc = new(gf, k, p)
    enc.Encode(sh)
    windows = (0, (1 << 31) - 4096, size - 4096)
    keep = {}
    for off in windows:
        win = [host(s[off:off + 4096]) for s in sh]
        want = [w.copy() for w in win]
        for i in range(k, k + p):
            want[i][:] = 0
        O.leo_encode(gf, k, p, want)
        for i in range(k, k + p):
            assert np.array_equal(win[i], want[i]), (gf, off, i)
        keep[off] = win
    cp = [None, sh[1], sh[2], sh[3], None, sh[5]]
    enc.Reconstruct(cp)
    for off in windows:
        assert np.array_equal(host(cp[0][off:off + 4096]), keep[off][0])
        assert np.array_equal(host(cp[4][off:off + 4096]), keep[off][4])
    del sh, cp
    torch.cuda.empty_cache()


@pytest.mark.parametrize("gf", [16, 8])
def test_errloc_cache_repeats_and_overflow(gf):
    """Error locators are cached per erasure pattern (at most 256): repeats
    hit the cache, patterns past the cap are computed per call, and every
    reconstruction stays bit-exact."""
    k, p, size = (40, 20, 128) if gf == 16 else (30, 10, 128)
    rng = np.random.default_rng(900 + gf)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
          [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(gf, k, p, ref) == 0
    enc = new(gf, k, p)
    lib = rs.lib()
    assert lib.rsgpu_leopard_errloc_cached(enc._h) == 0
    seen, pats = set(), []
    while len(pats) < 300:
        lost = tuple(sorted(int(x) for x in rng.choice(k + p, size=int(rng.integers(1, p + 1)), replace=False)))
        if lost not in seen:
            seen.add(lost)
            pats.append(lost)
    for rnd, batch in enumerate([pats, pats[:10], pats[-5:]]):
        for lost in batch:
            sh = [None if i in lost else dev(ref[i]) for i in range(k + p)]
            enc.Reconstruct(sh)
            for i in lost:
                assert np.array_equal(host(sh[i]), ref[i]), (rnd, lost, i)
        assert lib.rsgpu_leopard_errloc_cached(enc._h) == 256
    assert lib.rsgpu_leopard_errloc_cached(rs.New(4, 2)._h) == 0


@pytest.mark.parametrize("gf,k,p", [(16, 5, 3), (16, 7, 4), (8, 5, 3)])
def test_every_erasure_pattern_small_codes(gf, k, p):
    """Every set of up to p lost shards of a small Leopard code is rebuilt
    on the device byte for byte (the oracle recovers them all too)."""
    import itertools
    size = 128
    rng = np.random.default_rng(700 + 10 * gf + k)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_encode(gf, k, p, ref) == 0
    enc = new(gf, k, p)
    for e in range(1, p + 1):
        for lost in itertools.combinations(range(k + p), e):
            sh = [None if i in lost else dev(ref[i]) for i in range(k + p)]
            enc.Reconstruct(sh)
            for i in lost:
                assert np.array_equal(host(sh[i]), ref[i]), (lost, i)
