"""Generates the inline-PTX dispatch of the run-time-coefficient GF(2^8)
kernel (csrc/gf8_rt.cuh): one indirect jump (brx.idx over a branch-target
list) into 256 straight-line bodies, body c accumulating c * x into y on
bit-planes.

    python -m reedsolomon_b200.gen_rt_dispatch OUT.inc

Body c: multiplication by c in GF(2^8) (polynomial 0x11D, the reference's
field, galois.go) is linear over GF(2); plane b of c*x is the XOR of the
planes a of x for which bit b of c * 2^a is set.  The kernel precomputes,
per input, the XOR of every non-empty subset of its planes 0-3 (lo[m]) and of
planes 4-7 (hi[m]), m = 1..15 (22 XORs, shared by every output), so row b of
body c is one three-input XOR: y_b ^= lo[row_b & 15] ^ hi[row_b >> 4].
Operands of the asm statement: %0..%7 = y planes (read and written),
%8..%22 = lo[1..15], %23..%37 = hi[1..15], %38 = the coefficient (0..255).
Labels carry %= so every inlined copy is unique.

A C++ switch over the same 256 cases is compiled to a binary compare tree
(about nine compare-and-branch levels per dispatch); brx.idx is one jump.
"""
import os
import sys


def gf_mul(a, b):
    r = 0
    for _ in range(8):
        if b & 1:
            r ^= a
        b >>= 1
        a = ((a << 1) ^ (0x11D if a & 0x80 else 0)) & 0x1FF
    return r & 0xFF


def row_masks(c):
    """mask[b]: the planes of x that feed plane b of c*x."""
    cols = [gf_mul(c, 1 << a) for a in range(8)]
    return [sum(((cols[a] >> b) & 1) << a for a in range(8)) for b in range(8)]


def body(c):
    out = []
    for b, m in enumerate(row_masks(c)):
        lo, hi = m & 15, m >> 4
        if lo and hi:
            out.append("lop3.b32 %%%d, %%%d, %%%d, %%%d, 0x96;" % (b, b, 7 + lo, 22 + hi))
        elif lo or hi:
            out.append("xor.b32 %%%d, %%%d, %%%d;" % (b, b, 7 + lo if lo else 22 + hi))
    return out


def generate():
    lines = ["{", "rt_ts%=: .branchtargets " + ", ".join("rt_c%d_%%=" % c for c in range(256)) + ";",
             "brx.idx.uni %38, rt_ts%=;"]
    for c in range(256):
        lines.append("rt_c%d_%%=:" % c)
        lines += body(c)
        if c != 255:
            lines.append("bra.uni rt_end%=;")
    lines += ["rt_end%=:", "}"]
    text = "// Generated by reedsolomon_b200/gen_rt_dispatch.py; do not edit.\n"
    text += "#define RSGPU_RT_DISPATCH_ASM \\\n"
    text += " \\\n".join('    "%s\\n"' % l for l in lines) + "\n"
    return text


def write(path):
    text = generate()
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return path
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(text)
    os.replace(tmp, path)
    return path


if __name__ == "__main__":
    print(write(sys.argv[1]))
