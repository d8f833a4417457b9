"""StreamEncoder (streaming.go) over the device pipeline, against the oracle:
block-wise Encode / Verify / Reconstruct with file-like readers and writers,
short final blocks, mismatched sizes, reader/writer failures, Split/Join."""
import io

import numpy as np
import pytest

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu


def encoded(rng, k, p, size):
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.rs_encode(k, p, sh) == 0
    return sh


@pytest.mark.parametrize("k,p,size,block", [(10, 4, 100000, 16384), (6, 3, 4096, 4096), (17, 3, 1000, 64),
                                            (4, 2, 77777, 1 << 20), (40, 20, 5000, 1024)])
def test_stream_encode_verify_reconstruct(k, p, size, block):
    rng = np.random.default_rng(k * 7 + size)
    ref = encoded(rng, k, p, size)
    enc = rs.NewStream(k, p, rs.WithStreamBlockSize(block))
    outs = [io.BytesIO() for _ in range(p)]
    enc.Encode([io.BytesIO(ref[i].tobytes()) for i in range(k)], outs)
    for o in range(p):
        assert outs[o].getvalue() == ref[k + o].tobytes()
    assert enc.Verify([io.BytesIO(a.tobytes()) for a in ref])
    bad = [a.copy() for a in ref]
    bad[k][size - 1] ^= 1
    assert not enc.Verify([io.BytesIO(a.tobytes()) for a in bad])
    for data_only in (False, True):
        lost = sorted(int(x) for x in rng.choice(k + p, size=p, replace=False))
        valid = [None if i in lost else io.BytesIO(ref[i].tobytes()) for i in range(k + p)]
        fill = [io.BytesIO() if (i in lost and (i < k or not data_only)) else None for i in range(k + p)]
        enc.Reconstruct(valid, fill)
        for i in range(k + p):
            if fill[i] is not None:
                assert fill[i].getvalue() == ref[i].tobytes(), i


class _Failing(io.RawIOBase):
    def readinto(self, b):
        raise IOError("disk gone")


class _FailingWriter:
    def write(self, b):
        raise IOError("pipe closed")


def test_stream_errors():
    k, p, size = 5, 3, 3000
    rng = np.random.default_rng(4)
    ref = encoded(rng, k, p, size)
    enc = rs.NewStream(k, p, rs.WithStreamBlockSize(1024))
    with pytest.raises(rs.ErrShardNoData):
        enc.Encode([io.BytesIO(b"") for _ in range(k)], [io.BytesIO() for _ in range(p)])
    readers = [io.BytesIO(ref[i].tobytes()) for i in range(k)]
    readers[2] = io.BytesIO(ref[2].tobytes()[:1500])   # a short stream
    with pytest.raises(rs.ErrShardSize):
        enc.Encode(readers, [io.BytesIO() for _ in range(p)])
    readers = [io.BytesIO(ref[i].tobytes()) for i in range(k)]
    readers[3] = _Failing()
    with pytest.raises(rs.StreamReadError) as e:
        enc.Encode(readers, [io.BytesIO() for _ in range(p)])
    assert e.value.stream == 3
    writers = [io.BytesIO() for _ in range(p)]
    writers[1] = _FailingWriter()
    with pytest.raises(rs.StreamWriteError) as e:
        enc.Encode([io.BytesIO(ref[i].tobytes()) for i in range(k)], writers)
    assert e.value.stream == k + 1
    valid = [io.BytesIO(a.tobytes()) for a in ref]
    fill = [None] * (k + p)
    fill[0] = io.BytesIO()
    with pytest.raises(rs.ErrReconstructMismatch):
        enc.Reconstruct(valid, fill)
    too_few = [None] * (p + 1) + [io.BytesIO(ref[i].tobytes()) for i in range(p + 1, k + p)]
    with pytest.raises(rs.ErrTooFewShards):
        enc.Reconstruct(too_few, [io.BytesIO() if r is None else None for r in too_few])
    with pytest.raises(rs.ErrTooFewShards):
        enc.Encode([io.BytesIO()] * (k - 1), [io.BytesIO()] * p)


def test_stream_split_join():
    k, p = 6, 3
    enc = rs.NewStream(k, p)
    data = np.random.default_rng(8).integers(0, 256, 12345, dtype=np.uint8).tobytes()
    dst = [io.BytesIO() for _ in range(k)]
    enc.Split(io.BytesIO(data), dst, len(data))
    rc, want = O.split(k, p, np.frombuffer(data, np.uint8))
    for i in range(k):
        assert dst[i].getvalue() == want[i].tobytes()
    out = io.BytesIO()
    enc.Join(out, [io.BytesIO(d.getvalue()) for d in dst], len(data))
    assert out.getvalue() == data
    with pytest.raises(rs.ErrShortData):
        enc.Split(io.BytesIO(data[:100]), [io.BytesIO() for _ in range(k)], len(data))
    with pytest.raises(rs.ErrShortData):
        enc.Join(io.BytesIO(), [io.BytesIO(d.getvalue()) for d in dst], len(data) + 10**6)
