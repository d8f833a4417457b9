"""GPU parity tests of the classic GF(2^8) path against the CPU oracle.

Every check is bit-exact.  Small sizes compare whole outputs with the oracle;
the 64 MiB RS(10,4) case uses size-independent properties (encode -> erase ->
reconstruct round trips, verify) plus oracle windows (the code is bytewise,
so any column window of the full result must equal the oracle on that window).
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


def make(k, p, size, seed):
    data = O.seeded_shards(seed, k, size)
    return data + [np.zeros(size, np.uint8) for _ in range(p)]


def test_one_encode_kat(kats):
    oe = kats["one_encode"]
    enc = rs.New(oe["k"], oe["p"])
    sh = [dev(np.array(s, np.uint8)) for s in oe["shards"]]
    enc.Encode(sh)
    for i, v in oe["parity"].items():
        assert host(sh[int(i)]).tolist() == v
    assert enc.Verify(sh)
    sh[8][0] += 1
    assert not enc.Verify(sh)


def test_galois_slice_kats(kats):
    g = kats["galois"]
    inp = dev(np.array(g["in"], np.uint8))
    out = torch.zeros_like(inp)
    for s in g["slices"]:
        rs.gal_mul_slice(s["c"], inp, out, xor=s["xor"])
        assert host(out).tolist() == s["expect"]


def test_config1_rs10x3_1mib():
    """RS(10,3) x 1 MiB: Encode, Verify, erase {3,7,11}, Reconstruct; all bit-exact vs oracle."""
    k, p, size = 10, 3, 1 << 20
    ref = make(k, p, size, 1)
    assert O.rs_encode(k, p, ref) == 0
    enc = rs.New(k, p)
    sh = [dev(a) for a in make(k, p, size, 1)]
    enc.Encode(sh)
    for i in range(k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i
    assert enc.Verify(sh)
    for i in (3, 7, 11):
        sh[i] = None
    enc.Reconstruct(sh)
    for i in range(k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i


SWEEP = [(k, p) for k in (1, 2, 3, 5, 8, 10, 13, 17, 24, 32) for p in (1, 2, 3, 4, 5, 8)]
SIZES = [1, 15, 16, 17, 100, 4096 + 3, 65536 + 48]


@pytest.mark.parametrize("k,p", SWEEP)
def test_encode_sweep_vs_oracle(k, p):
    rng = np.random.default_rng(k * 64 + p)
    enc = rs.New(k, p)
    for size in SIZES:
        ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
              [np.zeros(size, np.uint8) for _ in range(p)]
        sh = [dev(a) for a in ref]
        assert O.rs_encode(k, p, ref) == 0
        enc.Encode(sh)
        for i in range(k, k + p):
            assert np.array_equal(host(sh[i]), ref[i]), (k, p, size, i)
        assert enc.Verify(sh)


@pytest.mark.parametrize("k,p", [(50, 20), (100, 20), (40, 17), (200, 56), (33, 3)])
def test_tiled_geometries_vs_oracle(k, p):
    """More than 32 inputs or 16 outputs: host tiling of the launch, with accumulate tiles."""
    size = 4096 + 64
    ref = make(k, p, size, k + p)
    assert O.rs_encode(k, p, ref) == 0
    enc = rs.New(k, p)
    sh = [dev(a) for a in make(k, p, size, k + p)]
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i
    assert enc.Verify(sh)
    sh[k + p - 1][5] ^= 1
    assert not enc.Verify(sh)
    sh[k + p - 1][5] ^= 1
    rng = np.random.default_rng(5)
    lost = rng.choice(k + p, size=p, replace=False)
    for i in lost:
        sh[int(i)] = None
    enc.Reconstruct(sh)
    for i in range(k + p):
        assert np.array_equal(host(sh[i]), ref[i]), i


@pytest.mark.parametrize("kind", ["cauchy", "par1", "jerasure"])
def test_matrix_options(kind):
    k, p, size = 8, 4, 10000
    ref = make(k, p, size, 9)
    assert O.rs_encode(k, p, ref, kind=kind) == 0
    enc = rs.New(k, p, {"cauchy": rs.WithCauchyMatrix, "par1": rs.WithPAR1Matrix,
                        "jerasure": rs.WithJerasureMatrix}[kind]())
    sh = [dev(a) for a in make(k, p, size, 9)]
    enc.Encode(sh)
    for i in range(k, k + p):
        assert np.array_equal(host(sh[i]), ref[i])


def test_misaligned_pointers_and_ranges():
    """codeSomeShards over [start, stop) with pointers at every 16-byte misalignment."""
    rng = np.random.default_rng(11)
    n_in, n_out, size = 7, 5, 5000
    rows = rng.integers(0, 256, (n_out, n_in), dtype=np.uint8)
    base_in = [rng.integers(0, 256, size + 64, dtype=np.uint8) for _ in range(n_in)]
    for shift in (0, 1, 3, 8, 15):
        ins_np = [a[shift:shift + size].copy() for a in base_in]
        want = [np.zeros(size, np.uint8) for _ in range(n_out)]
        O.code_some_shards(rows, ins_np, want)
        ins = [dev(a)[shift:shift + size] for a in base_in]
        outs_full = [torch.zeros(size + 64, dtype=torch.uint8, device="cuda") for _ in range(n_out)]
        outs = [o[shift:shift + size] for o in outs_full]
        rs.code_some_shards(rows, ins, outs)
        for o in range(n_out):
            assert np.array_equal(host(outs[o]), want[o]), shift
    # partial range, accumulate mode
    ins = [dev(a[:size]) for a in base_in]
    outs = [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(n_out)]
    start, stop = 37, 4001
    rs.code_some_shards(rows, ins, outs, clear=True, start=start, stop=stop)
    rs.code_some_shards(rows, ins, outs, clear=False, start=start, stop=stop)
    for o in range(n_out):
        assert not host(outs[o]).any()  # x ^ x == 0, untouched bytes stay 0


def test_check_some_shards_detects_every_position():
    rng = np.random.default_rng(2)
    k, p, size = 10, 4, 4096 + 7
    ref = make(k, p, size, 21)
    O.rs_encode(k, p, ref)
    enc = rs.New(k, p)
    sh = [dev(a) for a in ref]
    assert enc.Verify(sh)
    for pos in (0, 15, 16, 2048, size - 8, size - 1):
        for par in (k, k + p - 1):
            sh[par][pos] ^= 0x5A
            assert not enc.Verify(sh), (pos, par)
            sh[par][pos] ^= 0x5A
    assert enc.Verify(sh)


def test_reconstruct_variants_like_reference():
    """testReconstructData (reedsolomon_test.go:807-960) on the GPU."""
    k, p, size = 8, 5, 100000
    ref = make(k, p, size, 3)
    O.rs_encode(k, p, ref)
    enc = rs.New(k, p)
    sh = [dev(a) for a in ref]
    enc.Encode(sh)
    enc.ReconstructData(sh)  # all present: no-op
    cp = [sh[i] if i < k else None for i in range(k + p)]
    req = [False] * (k + p)
    req[10] = True
    enc.ReconstructSome(cp, req)
    assert np.array_equal(host(cp[10]), ref[10]) and cp[9] is None
    cp = list(sh)
    for i in (2, 3, 4, 5, 6):
        cp[i] = None
    req = [False] * k
    req[3] = req[4] = True
    enc.ReconstructSome(cp, req)
    assert np.array_equal(host(cp[3]), ref[3]) and np.array_equal(host(cp[4]), ref[4])
    assert cp[2] is None and cp[5] is None
    cp = list(sh)
    cp[0] = cp[2] = cp[12] = None
    enc.ReconstructData(cp)
    assert np.array_equal(host(cp[0]), ref[0]) and np.array_equal(host(cp[2]), ref[2]) and cp[12] is None
    cp = list(sh)
    for i in (0, 1, 9, 10, 11, 12):
        cp[i] = None
    with pytest.raises(rs.ErrTooFewShards):
        enc.ReconstructData(cp)
    with pytest.raises(rs.ErrTooFewShards):
        enc.ReconstructData([None])
    with pytest.raises(rs.ErrShardNoData):
        enc.ReconstructData([None] * (k + p))


def test_all_erasure_patterns_small():
    k, p, size = 6, 3, 777
    ref = make(k, p, size, 4)
    O.rs_encode(k, p, ref)
    enc = rs.New(k, p)
    base = [dev(a) for a in ref]
    import itertools
    for e in (1, 2, 3):
        for lost in itertools.combinations(range(k + p), e):
            sh = list(base)
            for i in lost:
                sh[i] = None
            enc.Reconstruct(sh)
            for i in lost:
                assert np.array_equal(host(sh[i]), ref[i]), lost


def test_encode_idx_equals_encode():
    k, p, size = 10, 4, 12345
    ref = make(k, p, size, 8)
    O.rs_encode(k, p, ref)
    enc = rs.New(k, p)
    parity = [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    for idx in range(k):
        enc.EncodeIdx(dev(ref[idx]), idx, parity)
    for o in range(p):
        assert np.array_equal(host(parity[o]), ref[k + o])


def test_errors():
    enc = rs.New(4, 2)
    sh = [torch.zeros(64, dtype=torch.uint8, device="cuda") for _ in range(6)]
    with pytest.raises(rs.ErrTooFewShards):
        enc.Encode(sh[:5])
    bad = list(sh)
    bad[2] = torch.zeros(63, dtype=torch.uint8, device="cuda")
    with pytest.raises(rs.ErrShardSize):
        enc.Encode(bad)
    with pytest.raises(rs.ErrShardNoData):
        enc.Encode([torch.zeros(0, dtype=torch.uint8, device="cuda")] * 6)
    with pytest.raises(rs.ErrInvShardNum):
        enc.EncodeIdx(sh[0], 4, sh[4:])


def test_host_path_encode_and_reconstruct():
    k, p, size = 10, 4, (3 << 20) + 48
    ref = make(k, p, size, 12)
    O.rs_encode(k, p, ref)
    enc = rs.New(k, p)
    hs = [torch.from_numpy(a.copy()).pin_memory() for a in make(k, p, size, 12)]
    enc.Encode(hs)
    for i in range(k, k + p):
        assert np.array_equal(hs[i].numpy(), ref[i])
    for i in (1, 5, 12):
        hs[i] = None
    enc.Reconstruct(hs)
    for i in (1, 5, 12):
        assert np.array_equal(hs[i].numpy(), ref[i])


def test_rs10x4_64mib_roundtrip_and_windows():
    """Full-size config: properties + oracle windows (bytewise code => windows are exact)."""
    k, p, size = 10, 4, 64 << 20
    g = torch.Generator(device="cuda").manual_seed(1234)
    sh = [torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g) for _ in range(k)]
    sh += [torch.empty(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    enc = rs.New(k, p)
    enc.Encode(sh)
    assert enc.Verify(sh)
    for off in (0, 12345 * 16, size - 65536):
        win = [host(s[off:off + 65536]) for s in sh]
        want = [w.copy() for w in win]
        for i in range(k, k + p):
            want[i][:] = 0
        O.rs_encode(k, p, want)
        for i in range(k, k + p):
            assert np.array_equal(win[i], want[i]), (off, i)
    rng = np.random.default_rng(99)
    orig = [s.clone() for s in sh]
    for _ in range(3):
        lost = rng.choice(k + p, size=p, replace=False)
        cp = list(sh)
        for i in lost:
            cp[int(i)] = None
        enc.Reconstruct(cp)
        for i in lost:
            assert torch.equal(cp[int(i)], orig[int(i)])


def test_shards_past_2gib_offsets():
    """Shards longer than 2^31 bytes (with a ragged tail for the byte kernel):
    byte offsets past the 32-bit range must address the right columns in
    encode, verify and reconstruct (oracle windows across the boundary)."""
    k, p = 3, 2
    size = (1 << 31) + 4096 + 48
    g = torch.Generator(device="cuda").manual_seed(77)
    sh = [torch.randint(0, 256, (size,), dtype=torch.uint8, device="cuda", generator=g) for _ in range(k)]
    sh += [torch.empty(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    enc = rs.New(k, p)
    enc.Encode(sh)
    assert enc.Verify(sh)
    windows = (0, (1 << 31) - 4096, size - 8192)
    for off in windows:
        win = [host(s[off:off + 8192]) for s in sh]
        want = [w.copy() for w in win]
        for i in range(k, k + p):
            want[i][:] = 0
        O.rs_encode(k, p, want)
        for i in range(k, k + p):
            assert np.array_equal(win[i], want[i]), (off, i)
    keep = {off: [host(s[off:off + 8192]) for s in sh] for off in windows}
    cp = [None, sh[1], sh[2], None, sh[4]]
    enc.Reconstruct(cp)
    for off in windows:
        assert np.array_equal(host(cp[0][off:off + 8192]), keep[off][0])
        assert np.array_equal(host(cp[3][off:off + 8192]), keep[off][3])
    del sh, cp
    torch.cuda.empty_cache()


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8])
def test_every_kernel_variant_bit_exact(variant):
    """Each variant of the GF(2^8) kernel (nibble-table address forms and the
    generated XOR network) gives the oracle's bytes."""
    lib = rs.lib()
    assert lib.rsgpu_force_variant(variant) == 0
    try:
        rng = np.random.default_rng(variant)
        for k, p, size in [(10, 4, 4096 * 3 + 16), (17, 3, 1000), (32, 16, 2048), (5, 9, 160), (3, 1, 64),
                           (6, 3, 65536 + 1024 + 5), (40, 20, 3072)]:
            ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
                  [np.zeros(size, np.uint8) for _ in range(p)]
            sh = [dev(a) for a in ref]
            O.rs_encode(k, p, ref)
            enc = rs.New(k, p)
            enc.Encode(sh)
            for i in range(k, k + p):
                assert np.array_equal(host(sh[i]), ref[i]), (variant, k, p, i)
            assert enc.Verify(sh)
            sh[k][size - 1] ^= 1
            assert not enc.Verify(sh)
            sh[k][size - 1] ^= 1
            sh[k + p - 1][0] ^= 0x80   # first chunk: inside the XOR network's range
            assert not enc.Verify(sh)
        if variant == 7 and lib.rsgpu_xornet_available():
            assert lib.rsgpu_xornet_sync() >= 1
    finally:
        lib.rsgpu_force_variant(-1)


def test_autotune_records_a_variant():
    import ctypes
    lib = rs.lib()
    ctx = rs.Context.get(0)
    ms = (ctypes.c_float * lib.rsgpu_num_variants())()
    best = ctypes.c_int(-1)
    assert lib.rsgpu_autotune_gf8(ctx.handle, 10, 4, 1 << 20, 0, 2, ms, ctypes.byref(best)) == 0
    assert 0 <= best.value < lib.rsgpu_num_variants()
    assert all(x > 0 for x in ms)
