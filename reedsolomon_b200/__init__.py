"""B200-native Reed-Solomon erasure coding behind klauspost/reedsolomon's Encoder interface.

The compute path is librsgpu.so (hand-written sm_100a kernels behind the
C-ABI in include/rsgpu.h); this package is its Python host mirror.
"""
from .encoder import *  # noqa: F401,F403
from .encoder import (New, Encoder, Context, RSError, code_some_shards, check_some_shards,  # noqa: F401
                      gal_mul_slice, slice_xor, build_matrix, invert_matrix, HostOnly,
                      autotune, record_variant, force_variant, generated_kernels_available,
                      wait_generated_kernels)
from ._lib import LIB_PATH, lib  # noqa: F401
