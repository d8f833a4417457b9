"""The oracle's opt-in AVX2 Leopard products (used only to time the CPU
baseline in bench.py) give the same bytes as its scalar restatement of
refMulAdd / refMul, the checker's path: encode and reconstruct of random
GF(2^16) and GF(2^8) geometries (shard sizes are multiples of 64 bytes in
both fields)."""
import numpy as np
import pytest

import oracle as O


def _run(gf, k, p, size, lost, simd):
    rng = np.random.default_rng(k * 1000 + p + size)
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8) for _ in range(p)]
    assert O.leo_simd(simd) == simd
    try:
        assert O.leo_encode(gf, k, p, sh) == 0
        enc = [s.copy() for s in sh]
        present = [0 if i in lost else 1 for i in range(k + p)]
        for i in lost:
            sh[i][:] = 0
        rc, _ = O.leo_reconstruct(gf, k, p, sh, present)
        assert rc == 0
        return enc, [s.copy() for s in sh]
    finally:
        O.leo_simd(False)


@pytest.mark.skipif(not O.leo_simd(True) or O.leo_simd(False), reason="needs AVX2")
@pytest.mark.parametrize("gf,k,p,size", [(16, 10, 4, 64), (16, 200, 100, 128), (16, 1000, 200, 192), (16, 3, 1, 640),
                                         (8, 10, 4, 64), (8, 100, 28, 128), (8, 192, 56, 192), (8, 5, 3, 320)])
def test_avx2_products_match_scalar(gf, k, p, size):
    rng = np.random.default_rng(gf + k + p)
    lost = sorted(rng.choice(k + p, size=p, replace=False).tolist())
    a_enc, a_rec = _run(gf, k, p, size, lost, False)
    b_enc, b_rec = _run(gf, k, p, size, lost, True)
    for i in range(k + p):
        assert np.array_equal(a_enc[i], b_enc[i]), ("encode", i)
        assert np.array_equal(a_rec[i], b_rec[i]), ("reconstruct", i)
