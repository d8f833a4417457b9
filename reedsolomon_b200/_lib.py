"""ctypes binding of librsgpu.so (the C-ABI declared in include/rsgpu.h).

The library is built in-tree by reedsolomon_b200.build; importing this module
never falls back to anything else: a missing or unloadable library raises.
"""
import atexit
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librsgpu.so")

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_voidp = ctypes.c_void_p
c_size = ctypes.c_size_t
# StreamEncoder callbacks (rsgpu_read_fn / rsgpu_write_fn)
READ_FN = ctypes.CFUNCTYPE(ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t)
WRITE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t)
c_int = ctypes.c_int
c_intp = ctypes.POINTER(ctypes.c_int)


class RsOptions(ctypes.Structure):
    _fields_ = [
        ("matrix_kind", c_int),
        ("fast_one_parity", c_int),
        ("leopard", c_int),
        ("inversion_cache", c_int),
        ("custom_matrix", c_voidp),
        ("custom_rows", c_int),
        ("custom_cols", c_int),
    ]


class RsStripe(ctypes.Structure):
    _fields_ = [
        ("op", c_int),
        ("data_shards", c_int),
        ("parity_shards", c_int),
        ("shard_size", c_size),
        ("shards", c_voidp),
        ("present", c_voidp),
    ]


class RsRequest(ctypes.Structure):
    _fields_ = [
        ("op", c_int),
        ("data_shards", c_int),
        ("parity_shards", c_int),
        ("leopard", c_int),
        ("shard_size", c_size),
        ("shards", c_voidp),
        ("present", c_voidp),
        ("tag", ctypes.c_uint64),
        ("result", c_int),
    ]


class RsCompletion(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("tag", ctypes.c_uint64), ("status", c_int),
                ("latency_us", ctypes.c_double), ("queue_us", ctypes.c_double)]


class RsServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("bytes", ctypes.c_double), ("elapsed_s", ctypes.c_double), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("max_inflight_bytes", ctypes.c_double)]


# name -> (restype, argtypes)
SIGNATURES = {
    "rsgpu_ctx_create": (c_int, [c_int, ctypes.POINTER(c_voidp)]),
    "rsgpu_ctx_destroy": (c_int, [c_voidp]),
    "rsgpu_ctx_set_stream": (c_int, [c_voidp, c_voidp]),
    "rsgpu_ctx_reset_stream": (c_int, [c_voidp]),
    "rsgpu_ctx_stream": (c_voidp, [c_voidp]),
    "rsgpu_ctx_synchronize": (c_int, [c_voidp]),
    "rsgpu_status_string": (ctypes.c_char_p, [c_int]),
    "rsgpu_last_error": (ctypes.c_char_p, []),
    "rsgpu_alloc_shards": (c_int, [c_voidp, c_int, c_size, c_voidp]),
    "rsgpu_free": (c_int, [c_voidp, c_voidp]),
    "rsgpu_host_alloc": (c_int, [c_size, ctypes.POINTER(c_voidp)]),
    "rsgpu_host_free": (c_int, [c_voidp]),
    "rsgpu_memcpy": (c_int, [c_voidp, c_voidp, c_size]),
    "rsgpu_options_init": (None, [ctypes.POINTER(RsOptions)]),
    "rsgpu_encoder_new": (c_int, [c_voidp, c_int, c_int, ctypes.POINTER(RsOptions), ctypes.POINTER(c_voidp)]),
    "rsgpu_encoder_free": (c_int, [c_voidp]),
    "rsgpu_encoder_info": (c_int, [c_voidp, c_intp, c_intp, c_intp, c_intp]),
    "rsgpu_encoder_matrix": (c_int, [c_voidp, c_voidp]),
    "rsgpu_encode": (c_int, [c_voidp, c_voidp, c_size]),
    "rsgpu_encode_idx": (c_int, [c_voidp, c_voidp, c_int, c_voidp, c_size]),
    "rsgpu_verify": (c_int, [c_voidp, c_voidp, c_size, c_intp]),
    "rsgpu_reconstruct": (c_int, [c_voidp, c_voidp, c_voidp, c_size, c_voidp]),
    "rsgpu_reconstruct_data": (c_int, [c_voidp, c_voidp, c_voidp, c_size, c_voidp]),
    "rsgpu_reconstruct_some": (c_int, [c_voidp, c_voidp, c_voidp, c_voidp, c_int, c_size, c_voidp]),
    "rsgpu_encode_async": (c_int, [c_voidp, c_voidp, c_size]),
    "rsgpu_reconstruct_async": (c_int, [c_voidp, c_voidp, c_voidp, c_size, c_int]),
    "rsgpu_encode_host": (c_int, [c_voidp, c_voidp, c_size]),
    "rsgpu_reconstruct_host": (c_int, [c_voidp, c_voidp, c_voidp, c_size, c_int, c_voidp]),
    "rsgpu_reconstruct_some_host": (c_int, [c_voidp, c_voidp, c_voidp, c_voidp, c_int, c_size, c_voidp]),
    "rsgpu_verify_host": (c_int, [c_voidp, c_voidp, c_size, c_intp]),
    "rsgpu_encode_idx_host": (c_int, [c_voidp, c_voidp, c_int, c_voidp, c_size]),
    "rsgpu_update_host": (c_int, [c_voidp, c_voidp, c_voidp, c_size]),
    "rsgpu_decode_idx_host": (c_int, [c_voidp, c_voidp, c_voidp, c_voidp, c_size]),
    "rsgpu_decode_plan": (c_int, [c_voidp, c_voidp, c_int, c_voidp, c_int, c_voidp, c_voidp, c_intp, c_voidp]),
    "rsgpu_code_some_shards": (c_int, [c_voidp, c_voidp, c_int, c_int, c_voidp, c_voidp, c_size, c_size, c_int]),
    "rsgpu_check_some_shards": (c_int, [c_voidp, c_voidp, c_int, c_int, c_voidp, c_voidp, c_size, c_intp]),
    "rsgpu_check_some_shards_noalloc": (c_int, [c_voidp, c_int, c_int, c_voidp, c_voidp, c_size, c_voidp, c_intp]),
    "rsgpu_gal_mul_slice": (c_int, [c_voidp, ctypes.c_uint8, c_voidp, c_voidp, c_size, c_int]),
    "rsgpu_slice_xor": (c_int, [c_voidp, c_voidp, c_voidp, c_size]),
    "rsgpu_autotune_gf8": (c_int, [c_voidp, c_int, c_int, c_size, c_int, c_int, c_voidp, c_intp]),
    "rsgpu_force_variant": (c_int, [c_int]),
    "rsgpu_num_variants": (c_int, []),
    "rsgpu_leopard_errloc_cached": (c_int, [c_voidp]),
    "rsgpu_record_variant": (c_int, [c_int, c_int, c_size, c_int, c_int]),
    "rsgpu_xornet_available": (c_int, []),
    "rsgpu_xornet_sync": (c_int, []),
    "rsgpu_xornet_drain": (c_int, []),
    "rsgpu_encoder_prepare_kernels": (c_int, [c_voidp]),
    "rsgpu_xornet_source": (ctypes.c_longlong, [c_voidp, c_int, c_int, c_int, c_int, c_int, ctypes.c_char_p,
                                                c_size]),
    "rsgpu_update": (c_int, [c_voidp, c_voidp, c_voidp, c_size]),
    "rsgpu_split_plan": (c_int, [c_voidp, c_size, c_size, c_voidp, c_voidp]),
    "rsgpu_split": (c_int, [c_voidp, c_voidp, c_size, c_size, c_voidp, c_size, c_voidp, c_voidp]),
    "rsgpu_join": (c_int, [c_voidp, c_voidp, c_voidp, c_size, c_size]),
    "rsgpu_stream_encode": (c_int, [c_voidp, READ_FN, WRITE_FN, c_voidp, c_size, c_voidp]),
    "rsgpu_stream_verify": (c_int, [c_voidp, READ_FN, c_voidp, c_size, c_voidp, c_voidp]),
    "rsgpu_stream_reconstruct": (c_int, [c_voidp, c_voidp, c_voidp, READ_FN, WRITE_FN, c_voidp, c_size, c_voidp]),
    "rsgpu_decode_idx": (c_int, [c_voidp, c_voidp, c_voidp, c_voidp, c_size]),
    "rsgpu_batch_create": (c_int, [c_voidp, c_voidp, ctypes.POINTER(c_voidp)]),
    "rsgpu_batch_destroy": (c_int, [c_voidp]),
    "rsgpu_batch_clear": (c_int, [c_voidp]),
    "rsgpu_batch_add": (c_int, [c_voidp, c_voidp, c_int]),
    "rsgpu_batch_run": (c_int, [c_voidp, c_int]),
    "rsgpu_batch_run_async": (c_int, [c_voidp, c_int]),
    "rsgpu_batch_results": (c_int, [c_voidp, c_intp, c_int]),
    "rsgpu_batch_info": (c_int, [c_voidp, c_intp, c_intp, ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_double)]),
    "rsgpu_batch_autotune": (c_int, [c_voidp, c_int, c_intp, c_intp, ctypes.POINTER(ctypes.c_float)]),
    "rsgpu_batch_set_tile": (c_int, [c_voidp, c_int]),
    "rsgpu_server_create": (c_int, [c_voidp, c_size, c_size, c_int, c_int, ctypes.POINTER(c_voidp)]),
    "rsgpu_server_submit": (c_int, [c_voidp, c_voidp, ctypes.POINTER(ctypes.c_uint64)]),
    "rsgpu_server_poll": (c_int, [c_voidp, c_voidp, c_int]),
    "rsgpu_server_release": (c_int, [c_voidp, ctypes.c_uint64]),
    "rsgpu_server_wait_idle": (c_int, [c_voidp, c_int]),
    "rsgpu_server_get_stats": (c_int, [c_voidp, c_voidp]),
    "rsgpu_server_reset_stats": (c_int, [c_voidp]),
    "rsgpu_server_replay": (c_int, [c_voidp, c_voidp, c_voidp, c_int, c_voidp]),
    "rsgpu_server_destroy": (c_int, [c_voidp]),
    "rsgpu_build_matrix": (c_int, [c_int, c_int, c_int, c_voidp]),
    "rsgpu_invert_matrix": (c_int, [c_voidp, c_int, c_voidp]),
    "rsgpu_gal_mul": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
}

_lib = None


def lib():
    """Load librsgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "librsgpu.so is missing at %s; build it with `python -m reedsolomon_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _lib = L
        # Background XOR-network compiles must not run into process teardown
        # (NVRTC's own exit handlers can run while one is in progress):
        # Python's atexit runs before any C-level exit handler.
        atexit.register(L.rsgpu_xornet_drain)
    return _lib


def ptr_array(ptrs):
    """Host array of device (or host) pointers, as the C-ABI's uint8_t** arguments."""
    arr = (c_voidp * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p if p else None
    return arr


def u8_array(vals):
    arr = (ctypes.c_uint8 * max(1, len(vals)))()
    for i, v in enumerate(vals):
        arr[i] = int(v)
    return arr
