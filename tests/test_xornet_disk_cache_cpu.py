"""Optional on-disk cache of the generated XOR-network kernels
(RSGPU_KERNEL_CACHE), on the CPU: a second process reads the cubins instead
of compiling them; a damaged file is ignored, recompiled and rewritten; with
the variable unset nothing is cached.  The harness
(tests/xornet_disk_cache.cpp) links the library's internal C++ entry points
and touches no GPU."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

import reedsolomon_b200 as rs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "reedsolomon_b200")
CUDA_INC = "/usr/local/cuda/include"


def _nvrtc():
    try:
        ctypes.CDLL("libnvrtc.so.12")
        return True
    except OSError:
        return False


pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                                reason="needs g++, CUDA headers and libnvrtc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    rs.lib()
    exe = tmp_path_factory.mktemp("xn") / "disk_cache"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                        "-I", CUDA_INC, os.path.join(HERE, "xornet_disk_cache.cpp"), "-o", str(exe),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG, "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


def run(exe, cache_dir):
    env = dict(os.environ)
    env.pop("RSGPU_KERNEL_CACHE", None)
    if cache_dir is not None:
        env["RSGPU_KERNEL_CACHE"] = str(cache_dir)
    r = subprocess.run([exe], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"compiles=(\d+) ok=(\d+)", r.stdout)
    return int(m.group(1)), int(m.group(2))


def test_second_process_reads_the_cache(harness, tmp_path):
    d = tmp_path / "kernels"
    n, ok = run(harness, d)
    assert ok == 3 and n >= 3
    files = sorted(p.name for p in d.iterdir())
    assert len(files) == 3 and all(f.startswith("rs_xornet_") and f.endswith(".cubin") for f in files)
    assert run(harness, d) == (0, 3)


def test_damaged_file_is_recompiled(harness, tmp_path):
    d = tmp_path / "kernels"
    run(harness, d)
    victim = sorted(d.iterdir())[0]
    data = victim.read_bytes()
    victim.write_bytes(data[: len(data) // 2])          # truncated
    n, ok = run(harness, d)
    assert ok == 3 and n >= 1
    assert victim.read_bytes() == data                  # rewritten whole
    victim.write_bytes(data + b"x")                      # trailing garbage
    n, ok = run(harness, d)
    assert ok == 3 and n >= 1
    flipped = bytearray(data)
    flipped[-100] ^= 0x04                                # a bit flipped inside the cubin
    victim.write_bytes(bytes(flipped))
    n, ok = run(harness, d)
    assert ok == 3 and n >= 1
    assert victim.read_bytes() == data
    assert run(harness, d) == (0, 3)


def test_cache_directory_is_private(harness, tmp_path):
    d = tmp_path / "kernels"
    run(harness, d)
    assert (os.stat(d).st_mode & 0o777) == 0o700


def test_no_cache_without_the_variable(harness, tmp_path):
    n, ok = run(harness, None)
    assert ok == 3 and n >= 3
