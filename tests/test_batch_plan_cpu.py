"""Work units of the persistent batch kernel (reedsolomon_b200/csrc/
batch_plan.h, used by batch.cu), compiled with g++ and run on the CPU over
3000 random job lists: boundaries cover the tiles in order, each unit's first
job holds its first tile, and no unit costs more than the average plus one
tile."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "reedsolomon_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_batch_unit_plan(tmp_path):
    exe = tmp_path / "batch_plan"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", CSRC, os.path.join(HERE, "batch_plan_harness.cpp"),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
