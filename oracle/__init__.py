"""ctypes binding of the CPU oracle (oracle.c / oracle_simd.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker / reference timing.  The product
(reedsolomon_b200) never imports it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None
c_voidp, c_int, c_size = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t

_SIGS = {
    "ora_gf8_tables": (None, [c_voidp] * 5),
    "ora_gf8_multable": (None, [c_voidp]),
    "ora_gal_mul": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
    "ora_gal_exp": (ctypes.c_uint8, [ctypes.c_uint8, c_int]),
    "ora_gal_divide": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
    "ora_gfni_matrix": (ctypes.c_uint64, [ctypes.c_uint8]),
    "ora_mat_invert": (c_int, [c_voidp, c_int, c_voidp]),
    "ora_mat_multiply": (None, [c_voidp, c_int, c_int, c_voidp, c_int, c_voidp]),
    "ora_build_matrix": (c_int, [c_int, c_int, c_int, c_voidp]),
    "ora_gal_mul_slice": (None, [ctypes.c_uint8, c_voidp, c_voidp, c_size, c_int]),
    "ora_code_some_shards": (None, [c_voidp, c_int, c_int, c_voidp, c_voidp, c_size, c_int]),
    "ora_rs_encode": (c_int, [c_int, c_int, c_int, c_voidp, c_size]),
    "ora_rs_encode_idx": (c_int, [c_int, c_int, c_int, c_voidp, c_int, c_voidp, c_size]),
    "ora_rs_update": (c_int, [c_int, c_int, c_int, c_voidp, c_voidp, c_size]),
    "ora_split": (c_int, [c_int, c_int, c_int, c_voidp, c_size, c_voidp, c_voidp]),
    "ora_join": (c_int, [c_int, c_voidp, c_voidp, c_int, c_voidp, c_size]),
    "ora_rs_decode_idx": (c_int, [c_int, c_int, c_int, c_voidp, c_voidp, c_voidp, c_size]),
    "ora_rs_verify": (c_int, [c_int, c_int, c_int, c_voidp, c_size, ctypes.POINTER(c_int)]),
    "ora_rs_reconstruct": (c_int, [c_int, c_int, c_int, c_voidp, c_voidp, c_size, c_int, c_voidp, c_int, c_voidp]),
    "ora_rs_decode_rows": (c_int, [c_int, c_int, c_int, c_voidp, c_int, c_voidp, c_int, c_voidp, c_voidp,
                                   ctypes.POINTER(c_int), c_voidp]),
    "ora_leo16_tables": (None, [c_voidp] * 4),
    "ora_leo16_mullog": (ctypes.c_uint16, [ctypes.c_uint16, ctypes.c_uint16]),
    "ora_leo_simd": (c_int, [c_int]),
    "ora_leo16_encode": (c_int, [c_int, c_int, c_voidp, c_size]),
    "ora_leo16_reconstruct": (c_int, [c_int, c_int, c_voidp, c_voidp, c_size, c_int, c_voidp]),
    "ora_leo16_errlocs": (c_int, [c_int, c_int, c_voidp, c_voidp]),
    "ora_leo16_verify": (c_int, [c_int, c_int, c_voidp, c_size, ctypes.POINTER(c_int)]),
    "ora_leo8_tables": (None, [c_voidp] * 4),
    "ora_leo8_mullog": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
    "ora_leo8_gfni_matrix": (ctypes.c_uint64, [ctypes.c_uint8]),
    "ora_leo8_encode": (c_int, [c_int, c_int, c_voidp, c_size]),
    "ora_leo8_reconstruct": (c_int, [c_int, c_int, c_voidp, c_voidp, c_size, c_int, c_voidp]),
    "ora_leo8_errlocs": (c_int, [c_int, c_int, c_voidp, c_voidp]),
    "ora_leo8_verify": (c_int, [c_int, c_int, c_voidp, c_size, ctypes.POINTER(c_int)]),
    "ora_simd_level": (c_int, []),
    "ora_code_some_shards_fast": (c_int, [c_voidp, c_int, c_int, c_voidp, c_voidp, c_size, c_int, c_int]),
}

MAT = {"default": 0, "cauchy": 1, "par1": 2, "jerasure": 3, "xor": 4}
# status codes of oracle.h (the reference's sentinel errors)
ERR = {"too_few_shards": -1, "shard_no_data": -2, "shard_size": -3, "invalid_shard_size": -4,
       "inv_shard_num": -5, "max_shard_num": -6, "not_supported": -7, "invalid_input": -8,
       "reconstruct_required": -9, "singular": -10, "not_square": -11, "short_data": -12}


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(_build.build())
        for n, (r, a) in _SIGS.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _rows_ptrs(arrs):
    a = (c_voidp * max(1, len(arrs)))()
    for i, x in enumerate(arrs):
        a[i] = None if x is None else x.ctypes.data
    return a


def _u8(vals):
    a = (ctypes.c_uint8 * max(1, len(vals)))()
    for i, v in enumerate(vals):
        a[i] = int(v)
    return a


def gf8_tables():
    log, exp, inv = (np.zeros(256, np.uint8) for _ in range(3))
    low, high = np.zeros(4096, np.uint8), np.zeros(4096, np.uint8)
    lib().ora_gf8_tables(log.ctypes.data, exp.ctypes.data, inv.ctypes.data, low.ctypes.data, high.ctypes.data)
    return log, exp, inv, low, high


def gf8_multable():
    m = np.zeros(65536, np.uint8)
    lib().ora_gf8_multable(m.ctypes.data)
    return m


def gal_mul(a, b):
    return lib().ora_gal_mul(a, b)


def gal_exp(a, n):
    return lib().ora_gal_exp(a, n)


def gfni_matrix(c):
    return lib().ora_gfni_matrix(c)


def invert(m):
    m = np.ascontiguousarray(m, np.uint8)
    out = np.zeros_like(m)
    rc = lib().ora_mat_invert(m.ctypes.data, m.shape[0], out.ctypes.data)
    return rc, out


def mat_multiply(a, b):
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    out = np.zeros((a.shape[0], b.shape[1]), np.uint8)
    lib().ora_mat_multiply(a.ctypes.data, a.shape[0], a.shape[1], b.ctypes.data, b.shape[1], out.ctypes.data)
    return out


def build_matrix(kind, k, total):
    out = np.zeros((total, k), np.uint8)
    rc = lib().ora_build_matrix(MAT[kind], k, total, out.ctypes.data)
    return rc, out


def gal_mul_slice(c, inp, out, xor=False):
    lib().ora_gal_mul_slice(c, inp.ctypes.data, out.ctypes.data, len(inp), int(xor))


def code_some_shards(rows, inputs, outputs, clear=True):
    rows = np.ascontiguousarray(rows, np.uint8)
    lib().ora_code_some_shards(rows.ctypes.data, rows.shape[1], rows.shape[0], _rows_ptrs(inputs),
                               _rows_ptrs(outputs), len(inputs[0]), int(clear))


def code_some_shards_fast(rows, inputs, outputs, clear=True, threads=1):
    rows = np.ascontiguousarray(rows, np.uint8)
    return lib().ora_code_some_shards_fast(rows.ctypes.data, rows.shape[1], rows.shape[0], _rows_ptrs(inputs),
                                           _rows_ptrs(outputs), len(inputs[0]), int(clear), threads)


def rs_encode(k, p, shards, kind="default"):
    return lib().ora_rs_encode(k, p, MAT[kind], _rows_ptrs(shards), len(shards[0]))


def rs_encode_idx(k, p, data, idx, parity, kind="default"):
    return lib().ora_rs_encode_idx(k, p, MAT[kind], data.ctypes.data, idx, _rows_ptrs(parity), len(data))


def split(k, p, data, leopard=False):
    """Split (reedsolomon.go:1803-1856, leopard.go:320-370): (rc, list of k+p shards)."""
    per = ctypes.c_size_t()
    rc = lib().ora_split(k, p, int(leopard), data.ctypes.data if len(data) else None, len(data), ctypes.byref(per), None)
    if rc:
        return rc, None
    out = np.zeros((k + p) * per.value, np.uint8)
    lib().ora_split(k, p, int(leopard), data.ctypes.data, len(data), ctypes.byref(per), out.ctypes.data)
    return 0, [out[i * per.value:(i + 1) * per.value] for i in range(k + p)]


def join(k, shards, out_size):
    """Join (reedsolomon.go:1858-1898): (rc, bytes)."""
    sizes = (ctypes.c_size_t * max(1, len(shards)))(*[0 if s is None else len(s) for s in shards])
    dst = np.zeros(max(1, out_size), np.uint8)
    rc = lib().ora_join(k, _rows_ptrs(shards), sizes, len(shards), dst.ctypes.data, out_size)
    return rc, (dst[:out_size] if rc == 0 else None)


def rs_update(k, p, shards, new_data, size, kind="default"):
    """Update (reedsolomon.go:762-853) in place; None entries are absent shards."""
    return lib().ora_rs_update(k, p, MAT[kind], _rows_ptrs(shards), _rows_ptrs(new_data), size)


def rs_decode_idx(k, p, dst, expect, inputs, size, kind="default"):
    """DecodeIdx (reedsolomon.go:1464-1617); expect=None selects merging mode."""
    return lib().ora_rs_decode_idx(k, p, MAT[kind], _rows_ptrs(dst), _u8(expect) if expect is not None else None,
                                   _rows_ptrs(inputs), size)


def rs_verify(k, p, shards, kind="default"):
    ok = c_int()
    rc = lib().ora_rs_verify(k, p, MAT[kind], _rows_ptrs(shards), len(shards[0]), ctypes.byref(ok))
    return rc, bool(ok.value)


def rs_reconstruct(k, p, shards, present, data_only=False, required=None, kind="default"):
    """shards: all k+p arrays allocated; present marks valid ones. Returns (rc, written)."""
    n = k + p
    written = (ctypes.c_uint8 * n)()
    req = _u8(required) if required is not None else None
    rc = lib().ora_rs_reconstruct(k, p, MAT[kind], _rows_ptrs(shards), _u8(present), len(shards[0]),
                                  int(data_only), req, len(required) if required is not None else 0, written)
    return rc, [bool(w) for w in written]


def rs_decode_rows(k, p, present, data_only=False, required=None, kind="default"):
    n = k + p
    rows = np.zeros((n, k), np.uint8)
    out_idx = (c_int * n)()
    in_idx = (c_int * k)()
    n_out = c_int()
    req = _u8(required) if required is not None else None
    rc = lib().ora_rs_decode_rows(k, p, MAT[kind], _u8(present), int(data_only), req,
                                  len(required) if required is not None else 0, rows.ctypes.data, out_idx,
                                  ctypes.byref(n_out), in_idx)
    no = n_out.value
    return rc, rows[:no].copy(), list(out_idx[:no]), (list(in_idx[:k]) if no else [])


def leo16_tables():
    log = np.zeros(65536, np.uint16)
    exp = np.zeros(65536, np.uint16)
    skew = np.zeros(65535, np.uint16)
    walsh = np.zeros(65536, np.uint16)
    lib().ora_leo16_tables(log.ctypes.data, exp.ctypes.data, skew.ctypes.data, walsh.ctypes.data)
    return log, exp, skew, walsh


def leo8_tables():
    log, exp, walsh = (np.zeros(256, np.uint8) for _ in range(3))
    skew = np.zeros(255, np.uint8)
    lib().ora_leo8_tables(log.ctypes.data, exp.ctypes.data, skew.ctypes.data, walsh.ctypes.data)
    return log, exp, skew, walsh


def leo_simd(on):
    """CPU-baseline timing only: AVX2 nibble-table products in the Leopard
    codec (True) or the scalar restatement (False, the checker's default).
    Returns whether the AVX2 path is on."""
    return bool(lib().ora_leo_simd(int(bool(on))))


def leo_encode(gf, k, p, shards):
    f = lib().ora_leo16_encode if gf == 16 else lib().ora_leo8_encode
    return f(k, p, _rows_ptrs(shards), len(shards[0]))


def leo_reconstruct(gf, k, p, shards, present, recover_all=True):
    f = lib().ora_leo16_reconstruct if gf == 16 else lib().ora_leo8_reconstruct
    n = k + p
    written = (ctypes.c_uint8 * n)()
    rc = f(k, p, _rows_ptrs(shards), _u8(present), len(shards[0]), int(recover_all), written)
    return rc, [bool(w) for w in written]


def leo_verify(gf, k, p, shards):
    f = lib().ora_leo16_verify if gf == 16 else lib().ora_leo8_verify
    ok = c_int()
    rc = f(k, p, _rows_ptrs(shards), len(shards[0]), ctypes.byref(ok))
    return rc, bool(ok.value)


def leo_errlocs(gf, k, p, present):
    if gf == 16:
        out = np.zeros(65536, np.uint16)
        lib().ora_leo16_errlocs(k, p, _u8(present), out.ctypes.data)
    else:
        out = np.zeros(256, np.uint8)
        lib().ora_leo8_errlocs(k, p, _u8(present), out.ctypes.data)
    return out


def simd_level():
    return lib().ora_simd_level()


def seeded_shards(seed, n, size):
    """Uniform random uint8 shards from a counter-based generator (numpy PCG64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(n)]
