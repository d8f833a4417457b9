"""Host-side algebra and planning of the product versus the oracle (CPU only)."""
import itertools

import numpy as np
import pytest

import oracle as O
import reedsolomon_b200 as rs


@pytest.mark.parametrize("kind", ["default", "cauchy", "par1", "jerasure"])
@pytest.mark.parametrize("k,p", [(1, 1), (5, 5), (10, 3), (10, 4), (17, 3), (32, 8), (100, 20), (200, 56)])
def test_build_matrix_matches_oracle(kind, k, p):
    rc, want = O.build_matrix(kind, k, k + p)
    assert rc == 0
    got = rs.build_matrix(kind, k, k + p)
    assert (got == want).all()


def test_jerasure_kat(kats):
    j = kats["jerasure"]
    m = rs.build_matrix("jerasure", j["k"], j["total"])
    assert m[j["k"]:].tolist() == j["parity_rows"]


def test_invert_kats(kats):
    for case in kats["matrix"]["inverse"]:
        inv = rs.invert_matrix(np.array(case["m"], np.uint8))
        assert str(inv.tolist()).replace(" ", "") == case["inverse"].replace(" ", "")
    for s in kats["matrix"]["singular"]:
        with pytest.raises(rs.ErrSingular):
            rs.invert_matrix(np.array(s, np.uint8))


def test_gal_mul_table():
    mt = O.gf8_multable().reshape(256, 256)
    lib = rs.lib()
    for a in range(0, 256, 7):
        for b in range(256):
            assert lib.rsgpu_gal_mul(a, b) == mt[a, b]


def _plans(k, p, rng, n=40):
    yield [1] * (k + p)
    for _ in range(n):
        e = rng.integers(1, p + 2)
        lost = set(rng.choice(k + p, size=min(e, k + p), replace=False).tolist())
        yield [0 if i in lost else 1 for i in range(k + p)]


@pytest.mark.parametrize("k,p", [(10, 3), (10, 4), (8, 5), (4, 2), (17, 3), (30, 8)])
def test_decode_plan_matches_oracle(k, p):
    rng = np.random.default_rng(k * 100 + p)
    enc = rs.New(k, p, rs.HostOnly())
    for present in _plans(k, p, rng):
        for data_only in (False, True):
            rc, rows, out_idx, in_idx = O.rs_decode_rows(k, p, present, data_only=data_only)
            if rc != 0:
                with pytest.raises(rs.RSError) as ei:
                    enc.DecodePlan(present, data_only)
                assert ei.value.code == rc
                continue
            got_rows, got_out, got_in = enc.DecodePlan(present, data_only)
            assert got_out == out_idx and got_in == in_idx
            assert (got_rows == rows).all()


def test_decode_plan_required():
    k, p = 8, 5
    enc = rs.New(k, p, rs.HostOnly())
    present = [1, 1, 0, 0, 0, 0, 0, 1] + [1] * 5
    req = [0, 0, 0, 1, 1, 0, 0, 0]
    rc, rows, oi, ii = O.rs_decode_rows(k, p, present, data_only=True, required=req)
    got = enc.DecodePlan(present, True, req)
    assert rc == 0 and got[1] == oi == [3, 4] and (got[0] == rows).all()
    # nothing required is missing -> nothing to do
    assert enc.DecodePlan(present, True, [1, 1, 0, 0, 0, 0, 0, 1])[1] == []


def test_inversion_cache_consistent():
    k, p = 10, 4
    a = rs.New(k, p, rs.HostOnly())
    b = rs.New(k, p, rs.HostOnly(), rs.WithInversionCache(False))
    for lost in itertools.combinations(range(k + p), 3):
        present = [0 if i in lost else 1 for i in range(k + p)]
        r1 = a.DecodePlan(present)
        r1b = a.DecodePlan(present)  # cached path
        r2 = b.DecodePlan(present)
        assert (r1[0] == r2[0]).all() and (r1b[0] == r2[0]).all()


def test_errors_mirror_reference():
    with pytest.raises(rs.ErrInvShardNum):
        rs.New(0, 1, rs.HostOnly())
    with pytest.raises(rs.ErrInvShardNum):
        rs.New(1, -1, rs.HostOnly())
    # too few present shards
    enc = rs.New(4, 2, rs.HostOnly())
    with pytest.raises(rs.ErrTooFewShards):
        enc.DecodePlan([1, 0, 0, 1, 1, 0])
    with pytest.raises(rs.ErrShardNoData):
        enc.DecodePlan([0] * 6)


def test_par1_singular_reported():
    # PAR1 matrices have singular sub-matrices (reedsolomon_test.go:158-176)
    k, p = 4, 4
    enc = rs.New(k, p, rs.HostOnly(), rs.WithPAR1Matrix())
    found = False
    for lost in itertools.combinations(range(k + p), p):
        present = [0 if i in lost else 1 for i in range(k + p)]
        rc = O.rs_decode_rows(k, p, present, kind="par1")[0]
        if rc == -10:
            found = True
            with pytest.raises(rs.ErrSingular):
                enc.DecodePlan(present)
    assert found


def test_custom_and_fast_one_parity_matrices():
    k = 6
    enc = rs.New(k, 1, rs.HostOnly(), rs.WithFastOneParityMatrix())
    assert (enc.Matrix()[k] == 1).all()
    cm = np.arange(2 * k, dtype=np.uint8).reshape(2, k) + 1
    enc = rs.New(k, 2, rs.HostOnly(), rs.WithCustomMatrix(cm))
    assert (enc.Matrix()[k:] == cm).all()


def test_codec_routing():
    assert rs.New(200, 57, rs.HostOnly()).codec == 1          # > 256 shards -> GF16
    assert rs.New(10, 4, rs.HostOnly(), rs.WithLeopardGF16()).codec == 1
    assert rs.New(10, 4, rs.HostOnly(), rs.WithLeopardGF()).codec == 2
    assert rs.New(10, 4, rs.HostOnly()).codec == 0
    assert rs.New(10, 4, rs.HostOnly()).ShardSizeMultiple() == 1
    assert rs.New(10, 4, rs.HostOnly(), rs.WithLeopardGF()).ShardSizeMultiple() == 64
