"""The timed configurations at full scale, checked byte for byte, through the
same code bench.py times: C2, RS(10,4) x 64 MiB with the 32 seeded
4-erasure patterns, Reconstruct and ReconstructData, before and after their
decode matrices' kernels are compiled, and through host buffers; and C3,
4096 stripes of mixed geometry (k in [4,32], p in [2,8], 4 KiB - 1 MiB)
encoded and reconstructed persistent, per stripe and as a graph, identical
across the three and equal to the oracle on a seeded sample.  The reference's
pattern: encode, delete, reconstruct, compare with the original bytes
(reedsolomon_test.go:306-418)."""
import os
import sys

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
import reedsolomon_b200 as rs  # noqa: E402

pytestmark = pytest.mark.gpu


def test_c2_reconstruct_32_patterns_64mib():
    k, p, S = bench.K_DATA, bench.P_PARITY, 64 << 20
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(5)
    shards = [torch.randint(0, 256, (S,), dtype=torch.uint8, device=dev, generator=g) for _ in range(k)]
    shards += [torch.empty(S, dtype=torch.uint8, device=dev) for _ in range(p)]
    enc = rs.New(k, p)
    enc.Encode(shards)
    assert enc.Verify(shards)
    enc.ctx.bind_current_stream()
    res = bench.extra_reconstruct(enc, rs.lib(), shards, S, torch.cuda.current_stream(dev), cpu_seconds=0.1)
    assert res["bit_exact"] and res["patterns"] == 32
    del shards
    torch.cuda.empty_cache()


def test_c3_batch_4096_stripes():
    res = bench.extra_batch(torch.device("cuda", 0), 4096, cpu_seconds=0.1)
    assert res["modes_identical"] and res["bit_exact"] and res["stripes"] == 4096
    torch.cuda.empty_cache()
