"""The bit-sliced GF(2^8) kernel with run-time coefficients (variant 8) on the
device, bit-exact with the oracle: every one of its 256 per-constant bodies,
every mode, several passes of outputs (more than 4), input tiles past 32,
sub-chunk tails, and the decode matrices of random erasure patterns (which
it runs without compiling anything per matrix)."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu

lib = rs.lib()
VARIANT = 8


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


class forced:
    def __enter__(self):
        assert lib.rsgpu_force_variant(VARIANT) == 0

    def __exit__(self, *exc):
        lib.rsgpu_force_variant(-1)


@pytest.mark.parametrize("mode", ["write", "xor", "verify"])
def test_every_coefficient_value(mode):
    """A 16 x 16 matrix holding each byte value once: all 256 bodies run, in
    four passes of four outputs."""
    rng = np.random.default_rng(5)
    rows = rng.permutation(256).astype(np.uint8).reshape(16, 16)
    size = 3 * 1024 + 48          # three whole chunks and a table-kernel tail
    ins = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(16)]
    base = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(16)]
    want = [b.copy() for b in base]
    O.code_some_shards(rows, ins, want, clear=(mode != "xor"))
    d_in = [dev(x) for x in ins]
    with forced():
        if mode == "verify":
            chk = [dev(w) for w in want]
            assert rs.check_some_shards(rows, d_in, chk)
            for o in (0, 7, 15):
                bad = [c.clone() for c in chk]
                bad[o][1024 + 513] ^= 0x10    # inside the bit-sliced chunks
                assert not rs.check_some_shards(rows, d_in, bad)
        else:
            d_out = [dev(b) for b in base]
            rs.code_some_shards(rows, d_in, d_out, clear=(mode == "write"))
            for o in range(16):
                assert np.array_equal(host(d_out[o]), want[o]), o


@pytest.mark.parametrize("k,p,size", [(10, 4, 1 << 20), (32, 8, 64 * 1024 + 64), (1, 1, 1024), (3, 13, 5000),
                                      (40, 6, 8192), (17, 3, 2 * 1024 * 1024 + 100)])
def test_encode_verify_geometries(k, p, size):
    rng = np.random.default_rng(k * 100 + p)
    ref = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + \
          [np.zeros(size, np.uint8) for _ in range(p)]
    O.rs_encode(k, p, ref)
    sh = [dev(r) for r in ref[:k]] + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    enc = rs.New(k, p)
    with forced():
        enc.Encode(sh)
        for i in range(k, k + p):
            assert np.array_equal(host(sh[i]), ref[i]), i
        assert enc.Verify(sh)
        sh[k + p - 1][0] ^= 1
        assert not enc.Verify(sh)


def test_decode_matrices_of_random_patterns():
    """RS(10,4) x 1 MiB reconstructs of random 4-erasure patterns
    (ReconstructData too) through variant 8 are bit-exact."""
    k, p, size = 10, 4, 1 << 20
    data = O.seeded_shards(31, k, size)
    ref = data + [np.zeros(size, np.uint8) for _ in range(p)]
    O.rs_encode(k, p, ref)
    full = [dev(r) for r in ref]
    enc = rs.New(k, p)
    rng = np.random.default_rng(8)
    with forced():
        for t in range(12):
            lost = sorted(rng.choice(k + p, size=4, replace=False).tolist())
            sh = [None if i in lost else full[i] for i in range(k + p)]
            if t % 2:
                enc.ReconstructData(sh)
                check = [i for i in lost if i < k]
            else:
                enc.Reconstruct(sh)
                check = lost
            for i in check:
                assert np.array_equal(host(sh[i]), ref[i]), (lost, i)
