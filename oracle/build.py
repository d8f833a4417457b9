"""Build recipe for the CPU oracle (test infrastructure, never shipped).

    python oracle/build.py          # -> oracle/liboracle.so

The reference (Go) cannot be compiled in this image (no Go toolchain), so
there is no oracle/_ref build; the restatement in oracle.c is the checker and
oracle_simd.c restates the reference's SIMD kernels for the timed CPU baseline.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "liboracle.so")
SRCS = ["oracle.c", "oracle_simd.c"]


def build(force=False):
    srcs = [os.path.join(HERE, s) for s in SRCS if os.path.exists(os.path.join(HERE, s))]
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "oracle.h")])
        if os.path.getmtime(OUT) >= newest:
            return OUT
    cmd = ["gcc", "-O3", "-std=gnu11", "-Wall", "-fPIC", "-shared", "-pthread", "-o", OUT] + srcs
    subprocess.check_call(cmd, cwd=HERE)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
