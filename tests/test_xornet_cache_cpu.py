"""Concurrency of the XOR-network compile cache, on the CPU: background
compiles queued through the launch path (which returns before any CUDA call
while a matrix is not compiled) race synchronous compiles of the same and of
new matrices; and compiles queued before fork() finish in both processes.
The harnesses (tests/xornet_cache_stress.cpp, tests/xornet_fork.cpp) link
the library's internal C++ entry points and must finish without deadlock."""
import ctypes
import os
import shutil
import subprocess
import sys

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


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                    reason="needs g++, CUDA headers and libnvrtc")
def test_sync_and_background_compiles_do_not_deadlock(tmp_path):
    rs.lib()  # built
    exe = tmp_path / "stress"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                        "-I", CUDA_INC, os.path.join(HERE, "xornet_cache_stress.cpp"), "-o", str(exe),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG, "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad=0" in r.stdout


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                    reason="needs g++, CUDA headers and libnvrtc")
def test_queued_compiles_survive_fork(tmp_path):
    rs.lib()
    exe = tmp_path / "fork"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                        "-I", CUDA_INC, os.path.join(HERE, "xornet_fork.cpp"), "-o", str(exe),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG, "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # own process group, so a hung child is killed with its parent
    p = subprocess.Popen([str(exe)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, start_new_session=True)
    try:
        out, err = p.communicate(timeout=300)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, 9)
        raise
    assert p.returncode == 0, out + err
    assert "child ok=1" in out and "child_status=0" in out


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                    reason="needs g++, CUDA headers and libnvrtc")
def test_exit_with_compiles_in_flight(tmp_path):
    """A process that exits while background compiles run exits cleanly
    (the workers are drained before NVRTC tears itself down)."""
    rs.lib()
    exe = tmp_path / "exit_queued"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                        "-I", CUDA_INC, os.path.join(HERE, "xornet_exit_queued.cpp"), "-o", str(exe),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG, "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    for args in ([], [], [], ["warm"], ["warm"], ["warm"]):
        r = subprocess.run([str(exe)] + args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0 and "queued" in r.stdout, (args, r.returncode, r.stderr[-2000:])


_PY_EXIT = """
import ctypes, sys, time
sys.path.insert(0, {root!r})
import reedsolomon_b200 as rs
rs.lib()
ctypes.CDLL({shim!r}).queue_compiles(0, 3)
time.sleep(0.05)
print("queued")
"""


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                    reason="needs g++, CUDA headers and libnvrtc")
def test_python_exit_with_compiles_in_flight(tmp_path):
    """A Python process that exits while its first background compiles run
    exits cleanly: the package drains them through atexit, before NVRTC's
    exit handlers (registered during its first compile) run.  Without that
    drain this exited with SIGSEGV in about half of the runs."""
    rs.lib()
    shim = tmp_path / "libexitshim.so"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-DRSGPU_EXIT_SHIM",
                        "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"), "-I", CUDA_INC,
                        os.path.join(HERE, "xornet_exit_queued.cpp"), "-o", str(shim),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    code = _PY_EXIT.format(root=ROOT, shim=str(shim))
    for _ in range(8):
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0 and "queued" in r.stdout, (r.returncode, r.stderr[-2000:])


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC) or not _nvrtc(),
                    reason="needs g++, CUDA headers and libnvrtc")
def test_compile_after_two_uses_and_lru_eviction(tmp_path):
    """A one-off matrix is not compiled; a second request queues it; at the
    cache's capacity new compiles evict the least recently used entries."""
    rs.lib()
    exe = tmp_path / "policy"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                        "-I", CUDA_INC, os.path.join(HERE, "xornet_policy.cpp"), "-o", str(exe),
                        "-L", PKG, "-lrsgpu", "-Wl,-rpath," + PKG, "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    env = dict(os.environ, RSGPU_XORNET_CACHE_CAP="3")
    env.pop("RSGPU_XORNET_MIN_USES", None)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
