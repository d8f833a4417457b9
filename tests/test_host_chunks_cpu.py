"""The host-buffer pipeline's column-chunk plan (reedsolomon_b200/csrc/
host_chunks.h, used by hostpath.cpp), compiled with g++ and run on the CPU:
exact plans for the documented cases and 200000 random ones covering
[0, size) with every chunk within the staging ring and every length but the
last a multiple of the codec's alignment."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "reedsolomon_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_chunk_plan(tmp_path):
    exe = tmp_path / "host_chunks"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", CSRC, os.path.join(HERE, "host_chunks_harness.cpp"),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
