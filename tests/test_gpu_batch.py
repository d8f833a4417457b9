"""Batched mixed-geometry execution versus the oracle and the per-stripe path."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu


def make_stripes(n, seed, ragged=False):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n):
        k = int(rng.integers(4, 33))
        p = int(rng.integers(2, 9))
        size = int(np.exp(rng.uniform(np.log(4096), np.log(262144)))) // 64 * 64
        if ragged and s % 7 == 3:
            size += 17  # not a multiple of 16: per-job fallback path
        data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
        ref = data + [np.zeros(size, np.uint8) for _ in range(p)]
        assert O.rs_encode(k, p, ref) == 0
        e = int(rng.integers(1, p + 1))
        lost = sorted(int(x) for x in rng.choice(k + p, size=e, replace=False))
        out.append((k, p, size, ref, lost))
    return out


@pytest.mark.parametrize("mode", ["persistent", "per_stripe", "graph"])
def test_batch_encode_verify_reconstruct(mode):
    stripes = make_stripes(48, 11, ragged=True)
    enc_b, ver_b, rec_b = rs.Batch(), rs.Batch(), rs.Batch()
    dev = []
    for (k, p, size, ref, lost) in stripes:
        sh = [torch.from_numpy(a).cuda() if i < k else torch.zeros(size, dtype=torch.uint8, device="cuda")
              for i, a in enumerate(ref)]
        dev.append(sh)
        enc_b.add_encode(k, p, sh)
        ver_b.add_verify(k, p, sh)
    enc_b.run(mode)
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        for i in range(k, k + p):
            assert np.array_equal(sh[i].cpu().numpy(), ref[i]), (k, p, size, i)
    ver_b.run(mode)
    assert all(ver_b.results())
    dev[5][stripes[5][0]][3] ^= 1
    ver_b.run(mode)
    res = ver_b.results()
    assert res[5] is False and all(r for i, r in enumerate(res) if i != 5)
    dev[5][stripes[5][0]][3] ^= 1
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        present = [0 if i in lost else 1 for i in range(k + p)]
        for i in lost:
            sh[i].zero_()
        rec_b.add_reconstruct(k, p, sh, present)
    rec_b.run(mode)
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        for i in lost:
            assert np.array_equal(sh[i].cpu().numpy(), ref[i]), (k, p, size, i)


@pytest.mark.parametrize("tile", [4096, 16384, 65536])
def test_batch_tile_sizes_identical(tile):
    stripes = make_stripes(24, 5)
    b = rs.Batch()
    b.set_tile(tile)
    dev = []
    for (k, p, size, ref, lost) in stripes:
        sh = [torch.from_numpy(a).cuda() if i < k else torch.zeros(size, dtype=torch.uint8, device="cuda")
              for i, a in enumerate(ref)]
        dev.append(sh)
        b.add_encode(k, p, sh)
    b.run("persistent")
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        for i in range(k, k + p):
            assert np.array_equal(sh[i].cpu().numpy(), ref[i])
    info = b.info()
    assert info["stripes"] == 24 and info["tiles"] > 0


def test_batch_data_only_and_errors():
    stripes = make_stripes(8, 3)
    b = rs.Batch()
    for (k, p, size, ref, lost) in stripes:
        sh = [torch.from_numpy(a).cuda() for a in ref]
        present = [0 if i in lost else 1 for i in range(k + p)]
        for i in lost:
            sh[i].zero_()
        b.add_reconstruct(k, p, sh, present, data_only=True)
        b.run()
        for i in lost:
            got = sh[i].cpu().numpy()
            if i < k:
                assert np.array_equal(got, ref[i])
            else:
                assert not got.any()  # ReconstructData leaves parity alone
        b = rs.Batch()
    with pytest.raises(rs.ErrTooFewShards):
        k, p, size, ref, lost = stripes[0]
        sh = [torch.from_numpy(a).cuda() for a in ref]
        rs.Batch().add_reconstruct(k, p, sh, [0] * (p + 1) + [1] * (k - 1))


def test_batch_autotune_keeps_outputs_exact():
    """The autotuner runs the batch's own jobs for each candidate shape; the
    chosen shape is kept, and outputs stay equal to the oracle's."""
    stripes = make_stripes(24, 23)
    enc_b = rs.Batch()
    dev = []
    for (k, p, size, ref, lost) in stripes:
        sh = [torch.from_numpy(a).cuda() if i < k else torch.zeros(size, dtype=torch.uint8, device="cuda")
              for i, a in enumerate(ref)]
        dev.append(sh)
        enc_b.add_encode(k, p, sh)
    tile, ctas, ms = enc_b.autotune(reps=1)
    assert tile in (4096, 8192, 16384, 32768, 65536) and ctas in (2, 3, 4) and ms > 0
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        for i in range(k, k + p):
            sh[i].zero_()
    enc_b.run("persistent")
    for (k, p, size, ref, lost), sh in zip(stripes, dev):
        for i in range(k, k + p):
            assert np.array_equal(sh[i].cpu().numpy(), ref[i]), (k, p, size, i)
