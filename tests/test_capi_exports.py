"""The C-ABI library loads and exports every function include/rsgpu.h declares (CPU only)."""
import ctypes
import os
import re

import reedsolomon_b200
from reedsolomon_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(rsgpu_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "rsgpu_encode" in names and "rsgpu_code_some_shards" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(reedsolomon_b200.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_status_strings():
    lib = _lib.lib()
    assert lib.rsgpu_status_string(-1) == b"too few shards given"
    assert lib.rsgpu_status_string(-10) == b"matrix is singular"
