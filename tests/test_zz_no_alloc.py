"""rsgpu_check_some_shards_noalloc: parity verification without device allocation.

Callers that cannot allocate device memory when they verify (a process that
reserved its whole HBM budget up front, a latency-critical path that must not
risk cudaMalloc) use this entry point; its scratch is a static 8 MiB array per
device.  These checks compare it with the regular rsgpu_check_some_shards on
the same inputs, two calls in a row (the static flag must be cleared between
calls), with and without a corrupted parity byte.  This file is collected
last so a stop-at-first-failure run has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs
from reedsolomon_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _both(rows, ins, chk):
    """(regular result, no-alloc result) for the same inputs."""
    lib = L.lib()
    ctx = rs.Context.get(0)
    ctx.bind_current_stream()
    rows = np.ascontiguousarray(rows, np.uint8)
    n_out, n_in = rows.shape
    pi = L.ptr_array([t.data_ptr() for t in ins])
    pc = L.ptr_array([t.data_ptr() for t in chk])
    ok_a, ok_b = ctypes.c_int(-1), ctypes.c_int(-1)
    assert lib.rsgpu_check_some_shards(ctx.handle, rows.ctypes.data, n_in, n_out, pi, pc, len(ins[0]),
                                       ctypes.byref(ok_a)) == 0
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.rsgpu_check_some_shards_noalloc(rows.ctypes.data, n_in, n_out, pi, pc, len(ins[0]),
                                             ctypes.c_void_p(stream), ctypes.byref(ok_b))
    assert rc == 0, lib.rsgpu_last_error()
    return bool(ok_a.value), bool(ok_b.value)


@pytest.mark.parametrize("k,p,size", [(10, 4, (1 << 20) + 16), (5, 3, 1000), (40, 6, 65536)])
def test_noalloc_matches_regular_verify_twice(k, p, size):
    _, m = O.build_matrix("default", k, k + p)
    rows = m[k:]
    data = O.seeded_shards(k * 7 + p, k, size)
    par = [np.zeros(size, np.uint8) for _ in range(p)]
    O.code_some_shards(rows, data, par)
    ins = [torch.from_numpy(d).cuda() for d in data]
    chk = [torch.from_numpy(x).cuda() for x in par]
    for _ in range(2):
        assert _both(rows, ins, chk) == (True, True)
    chk[p - 1][size // 2] ^= 0x40
    for _ in range(2):
        assert _both(rows, ins, chk) == (False, False)
    chk[p - 1][size // 2] ^= 0x40
    for _ in range(2):  # a stale mismatch flag from the previous calls must not leak
        assert _both(rows, ins, chk) == (True, True)


def test_noalloc_rejects_scratch_overflow():
    lib = L.lib()
    k, p, size = 40, 4, 4 << 20  # 4 partial rows of 4 MiB > 8 MiB of static scratch
    rows = np.ones((p, k), np.uint8)
    ins = [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(k)]
    chk = [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
    ok = ctypes.c_int(-1)
    rc = lib.rsgpu_check_some_shards_noalloc(rows.ctypes.data, k, p, L.ptr_array([t.data_ptr() for t in ins]),
                                             L.ptr_array([t.data_ptr() for t in chk]), size,
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                             ctypes.byref(ok))
    assert rc == -8
    assert b"8 MiB" in lib.rsgpu_last_error()


def test_noalloc_runs_table_kernels_only():
    """Large shards default to kernels compiled at run time, whose first
    launch loads a module (a device allocation): the no-alloc entry point
    must never queue or load one, even with that variant forced."""
    lib = L.lib()
    rng = np.random.default_rng(77)
    k, p, size = 6, 3, 512 << 10
    rows = rng.integers(1, 256, (p, k), dtype=np.uint8)   # a matrix no other test uses
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    par = [np.zeros(size, np.uint8) for _ in range(p)]
    O.code_some_shards(rows, data, par)
    ins = [torch.from_numpy(d).cuda() for d in data]
    chk = [torch.from_numpy(x).cuda() for x in par]
    pi = L.ptr_array([t.data_ptr() for t in ins])
    pc = L.ptr_array([t.data_ptr() for t in chk])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    before = lib.rsgpu_xornet_sync()
    for forced in (-1, 7):
        assert lib.rsgpu_force_variant(forced) == 0
        try:
            for _ in range(2):
                ok = ctypes.c_int(-1)
                assert lib.rsgpu_check_some_shards_noalloc(rows.ctypes.data, k, p, pi, pc, size, stream,
                                                           ctypes.byref(ok)) == 0
                assert ok.value == 1
        finally:
            lib.rsgpu_force_variant(-1)
    assert lib.rsgpu_xornet_sync() == before


def test_noalloc_allocates_nothing_after_first_call():
    """Once the first call has set a device up, further calls of every shape
    (tails, 16 outputs, more than 32 inputs) leave the device's free memory
    exactly as it was: nothing is allocated and no code is loaded."""
    lib = L.lib()
    rng = np.random.default_rng(91)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    calls = []
    for k, p, size in [(10, 4, (1 << 20) + 16), (5, 3, 1000), (40, 6, 65536), (3, 1, 64), (32, 16, 4096),
                       (17, 3, 12345), (64, 2, 100000)]:
        rows = rng.integers(0, 256, (p, k), dtype=np.uint8)
        data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
        par = [np.zeros(size, np.uint8) for _ in range(p)]
        O.code_some_shards(rows, data, par)
        ins = [torch.from_numpy(d).cuda() for d in data]
        chk = [torch.from_numpy(x).cuda() for x in par]
        calls.append((rows, k, p, ins, chk, L.ptr_array([t.data_ptr() for t in ins]),
                      L.ptr_array([t.data_ptr() for t in chk]), size))

    def run(c):
        rows, k, p, _, _, pi, pc, size = c
        ok = ctypes.c_int(-1)
        assert lib.rsgpu_check_some_shards_noalloc(rows.ctypes.data, k, p, pi, pc, size, stream,
                                                   ctypes.byref(ok)) == 0, lib.rsgpu_last_error()
        return ok.value

    assert run(calls[0]) == 1  # set-up call of this test (the device may already be set up)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        for c in calls:
            assert run(c) == 1
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
