"""The generated dispatch of the run-time-coefficient GF(2^8) kernel
(reedsolomon_b200/gen_rt_dispatch.py), checked on the CPU: every body c,
executed instruction by instruction on bit-planes, accumulates exactly
c * x for every byte x (against the oracle's field product, pinned to the
reference's tables), and the branch-target list names the 256 bodies in
coefficient order."""
import re

import oracle as O
from reedsolomon_b200 import gen_rt_dispatch as G


def _bodies():
    text = G.generate()
    lines = [l.strip().rstrip("\\").strip()[1:-3] for l in text.splitlines()[2:]]
    bodies, cur = {}, None
    for l in lines:
        m = re.match(r"rt_c(\d+)_%=:$", l)
        if m:
            cur = int(m.group(1))
            bodies[cur] = []
        elif cur is not None and (l.startswith("lop3") or l.startswith("xor")):
            bodies[cur].append(l)
    return text, bodies


def _run(body, x):
    """y = 0; execute body with operands %0..%7 = y planes, %8..%22 = lo[1..15],
    %23..%37 = hi[1..15] (XORs of subsets of the low / high four planes of
    x, as the kernel builds them); x is one byte, its planes are its bits.
    Returns the y byte."""
    bits = [(x >> a) & 1 for a in range(8)]
    lo = [0] * 16
    hi = [0] * 16
    for m in range(16):
        for a in range(4):
            if (m >> a) & 1:
                lo[m] ^= bits[a]
                hi[m] ^= bits[4 + a]
    reg = [0] * 8 + lo[1:] + hi[1:]
    for ins in body:
        ops = [int(v) for v in re.findall(r"%(\d+)", ins)]
        if ins.startswith("lop3"):
            assert ins.endswith("0x96;")
            d, a, b, c = ops
            reg[d] = reg[a] ^ reg[b] ^ reg[c]
        else:
            d, a, b = ops
            reg[d] = reg[a] ^ reg[b]
    return sum(reg[b] << b for b in range(8))


def test_every_body_multiplies():
    text, bodies = _bodies()
    assert sorted(bodies) == list(range(256))
    for c in range(256):
        assert all(_run(bodies[c], x) == O.gal_mul(c, x) for x in range(256)), c
        assert len(bodies[c]) <= 8
    assert bodies[0] == []


def test_branch_targets_in_coefficient_order():
    text = G.generate()
    m = re.search(r"\.branchtargets ([^;]+);", text)
    labels = [t.strip() for t in m.group(1).split(",")]
    assert labels == ["rt_c%d_%%=" % c for c in range(256)]
    assert "brx.idx.uni %38" in text
