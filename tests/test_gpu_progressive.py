"""GPU parity of the progressive entry points against the oracle:
Update (reedsolomon.go:762-853) and DecodeIdx (reedsolomon.go:1464-1617)."""
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


def encoded(rng, k, p, size):
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.rs_encode(k, p, sh) == 0
    return sh


@pytest.mark.parametrize("k,p,size,changed", [(10, 4, 4096, (1, 7)), (6, 3, 1000, (0,)), (17, 3, 65536 + 48, (2, 5, 16)),
                                              (40, 8, 2048, tuple(range(0, 40, 3))), (5, 1, 333, (4,))])
def test_update_matches_oracle(k, p, size, changed):
    rng = np.random.default_rng(k * 100 + p)
    ref = encoded(rng, k, p, size)
    new = [None] * k
    for c in changed:
        new[c] = rng.integers(0, 256, size, dtype=np.uint8)
    want = [a.copy() for a in ref]
    assert O.rs_update(k, p, want, new, size) == 0
    sh = [dev(a) for a in ref]
    rs.New(k, p).Update(sh, [None if x is None else dev(x) for x in new])
    for i in range(k + p):
        assert np.array_equal(host(sh[i]), want[i]), i
    # parity equals a fresh encode of the new data
    fresh = [a.copy() for a in ref]
    for c in changed:
        fresh[c] = new[c]
    O.rs_encode(k, p, fresh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), fresh[i])


def test_update_errors():
    k, p, size = 6, 3, 256
    rng = np.random.default_rng(1)
    sh = [dev(a) for a in encoded(rng, k, p, size)]
    enc = rs.New(k, p)
    with pytest.raises(rs.ErrShardNoData):
        enc.Update(sh, [None] * k)
    with pytest.raises(rs.ErrTooFewShards):
        enc.Update(sh[:-1], [None] * k)
    new = [None] * k
    new[2] = dev(rng.integers(0, 256, size, dtype=np.uint8))
    missing = list(sh)
    missing[2] = None
    with pytest.raises(rs.ErrInvalidInput):
        enc.Update(missing, new)
    nopar = list(sh)
    nopar[k] = None
    with pytest.raises(rs.ErrInvalidInput):
        enc.Update(nopar, new)
    with pytest.raises(rs.ErrNotSupported):
        rs.New(k, p, rs.WithLeopardGF16()).Update(sh, new)


@pytest.mark.parametrize("k,p,size", [(10, 4, 4096), (6, 3, 1000), (17, 3, 65536 + 48), (40, 8, 2048)])
def test_decode_idx_progressive_matches_oracle(k, p, size):
    rng = np.random.default_rng(k + p + size)
    ref = encoded(rng, k, p, size)
    n = k + p
    for trial in range(3):
        lost = set(int(x) for x in rng.choice(n, size=p, replace=False))
        extra = set() if trial == 0 else {int(x) for x in rng.choice(sorted(lost), size=1)}
        expect = [0 if i in lost and i not in extra else 1 for i in range(n)]
        # two partial decoders fed disjoint input batches, then merged
        want_a = [None if expect[i] else np.zeros(size, np.uint8) for i in range(n)]
        want_b = [None if expect[i] else np.zeros(size, np.uint8) for i in range(n)]
        got_a = [None if expect[i] else torch.zeros(size, dtype=torch.uint8, device="cuda") for i in range(n)]
        got_b = [None if expect[i] else torch.zeros(size, dtype=torch.uint8, device="cuda") for i in range(n)]
        order = [i for i in range(n) if expect[i]]
        rng.shuffle(order)
        half = len(order) // 2
        enc = rs.New(k, p)
        for batch, want, got in ((order[:half], want_a, got_a), (order[half:], want_b, got_b)):
            for chunk in np.array_split(np.array(batch, dtype=int), 2):
                inp_h = [ref[i] if i in chunk else None for i in range(n)]
                inp_d = [dev(ref[i]) if i in chunk else None for i in range(n)]
                assert O.rs_decode_idx(k, p, want, expect, inp_h, size) == 0
                enc.DecodeIdx(got, expect, inp_d)
        for i in range(n):
            if want_a[i] is not None:
                assert np.array_equal(host(got_a[i]), want_a[i])
                assert np.array_equal(host(got_b[i]), want_b[i])
        assert O.rs_decode_idx(k, p, want_a, None, want_b, size) == 0
        enc.DecodeIdx(got_a, None, got_b)
        for i in range(n):
            if want_a[i] is not None:
                assert np.array_equal(host(got_a[i]), want_a[i])
                assert np.array_equal(want_a[i], ref[i])  # the merged result is the lost shard


def test_decode_idx_errors():
    k, p, size = 6, 3, 128
    rng = np.random.default_rng(2)
    ref = [dev(a) for a in encoded(rng, k, p, size)]
    enc = rs.New(k, p)
    n = k + p
    expect = [1] * k + [0] * p
    dst = [None] * k + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    bad = [None] * n
    bad[k] = ref[k]
    with pytest.raises(rs.ErrInvalidInput):
        enc.DecodeIdx(dst, expect, bad)                      # input not marked as expected
    with pytest.raises(rs.ErrInvalidInput):
        enc.DecodeIdx([ref[0]] + dst[1:], expect, [None] * n)  # dst for an expected shard
    with pytest.raises(rs.ErrTooFewShards):
        enc.DecodeIdx([None] * 3 + [torch.zeros(size, dtype=torch.uint8, device="cuda")] * (n - 3),
                      [1, 1, 1] + [0] * (n - 3), [None] * n)
    with pytest.raises(rs.ErrInvalidShardSize):
        enc.DecodeIdx(dst, expect, [ref[0][:64]] + [None] * (n - 1))
    with pytest.raises(rs.ErrInvalidInput):
        enc.DecodeIdx(dst, expect[:-1], [None] * n)
    with pytest.raises(rs.ErrNotSupported):
        rs.New(k, p, rs.WithLeopardGF16()).DecodeIdx(dst, expect, [None] * n)


def test_update_full_size_round_trip():
    """RS(10,4) x 64 MiB: update two data shards, then Verify against the new data."""
    k, p, size = 10, 4, 64 << 20
    g = torch.Generator(device="cuda").manual_seed(5)
    sh = [torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g) for _ in range(k)]
    sh += [torch.empty(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    enc = rs.New(k, p)
    enc.Encode(sh)
    new = [None] * k
    new[3] = torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g)
    new[8] = torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g)
    old3 = sh[3].clone()
    enc.Update(sh, new)
    assert torch.equal(sh[3], old3 ^ new[3])
    fresh = list(sh)
    fresh[3], fresh[8] = new[3], new[8]
    assert enc.Verify(fresh)
