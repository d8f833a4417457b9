"""Extract the reference's own known-answer vectors into tests/golden/reference_kats.json.

Run once in a container that has the reference checkout (read as text only,
nothing is executed):

    python tests/golden/make_golden.py /path/to/klauspost/reedsolomon

Sources (paths inside the reference project):
  galois.go            logTable :29, expTable :71, invTable :78, mulTable :80,
                       mulTableLow :337, mulTableHigh :593, gf2p811dMulMatrices :948
  leopard8.go          gf2p811dMulMatricesLeo8 :1271
  galois_test.go       testGalois :127-174 (galMultiply / galMulSlice(Xor) / galExp KATs)
  reedsolomon_test.go  TestOneEncode :1075-1125, TestBuildMatrixJerasure :129-156
  matrix_test.go       TestMatrixMultiply :91-115, TestMatrixInverse :118-217
  leopard_test.go      TestAddMod :167-190;  leopard8_test.go TestAddMod8 :10-33

The large mulTable is stored as a SHA-256 of its 65536 bytes; everything else
is stored verbatim.  The committed JSON travels with the repository; nothing
at test time reads the reference checkout.
"""
import hashlib
import json
import os
import re
import sys


def _braced_block(src, start):
    """Return the text between the '{' at/after start and its matching '}'."""
    i = src.index("{", start)
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i + 1:j]
    raise ValueError("unbalanced braces")


def _ints(text):
    return [int(t, 0) for t in re.findall(r"0x[0-9a-fA-F]+|\d+", text)]


def _var_table(src, name):
    m = re.search(r"var\s+%s\s*=\s*\[[^\]]*\]" % re.escape(name), src)
    if not m:
        raise KeyError(name)
    # skip the type (e.g. [256][16]uint8) to reach the composite literal
    body_start = src.index("{", m.end())
    return _ints(_braced_block(src, body_start - 1))


def _func_body(src, name):
    m = re.search(r"func\s+%s\s*\(" % re.escape(name), src)
    if not m:
        raise KeyError(name)
    # body starts at the first '{' after the closing ')' of the signature line
    line_end = src.index("\n", m.end())
    brace = src.rindex("{", m.end(), line_end + 1)
    return _braced_block(src, brace)


def galois_tables(ref):
    src = open(os.path.join(ref, "galois.go")).read()
    out = {
        "logTable": _var_table(src, "logTable"),
        "expTable": _var_table(src, "expTable"),
        "invTable": _var_table(src, "invTable"),
        "mulTableLow": _var_table(src, "mulTableLow"),
        "mulTableHigh": _var_table(src, "mulTableHigh"),
        "gf2p811dMulMatrices": _var_table(src, "gf2p811dMulMatrices"),
    }
    mt = _var_table(src, "mulTable")
    assert len(mt) == 65536
    out["mulTable_sha256"] = hashlib.sha256(bytes(mt)).hexdigest()
    assert len(out["logTable"]) == 256 and len(out["expTable"]) == 256
    assert len(out["mulTableLow"]) == 4096 and len(out["mulTableHigh"]) == 4096
    assert len(out["gf2p811dMulMatrices"]) == 256
    src8 = open(os.path.join(ref, "leopard8.go")).read()
    out["gf2p811dMulMatricesLeo8"] = _var_table(src8, "gf2p811dMulMatricesLeo8")
    assert len(out["gf2p811dMulMatricesLeo8"]) == 256
    return out


def galois_kats(ref):
    body = _func_body(open(os.path.join(ref, "galois_test.go")).read(), "testGalois")
    kats = {"mul": [], "exp": [], "slices": []}
    for a, b, r in re.findall(r"galMultiply\((\d+),\s*(\d+)\)\s*!=\s*(\d+)", body):
        kats["mul"].append([int(a), int(b), int(r)])
    for a, n, r in re.findall(r"galExp\((\d+),\s*(\d+)\)\s*!=\s*(\d+)", body):
        kats["exp"].append([int(a), int(n), int(r)])
    inp = _ints(re.search(r"in := \[\]byte\{([^}]*)\}", body).group(1))
    kats["in"] = inp
    # Walk the body in source order: literals assign expect/expectXor, calls
    # set the pending coefficient, and each bytes.Compare(out, NAME) closes a KAT.
    tok = re.compile(r"(expect(?:Xor)?)\s*:?=\s*\[\]byte\{([^}]*)\}"
                     r"|galMulSlice(Xor)?\((\d+),\s*in,\s*out"
                     r"|bytes\.Compare\(out,\s*(expect(?:Xor)?)\)")
    values, call = {}, None
    for name, lit, xor, coef, cmp_name in tok.findall(body):
        if name:
            values[name] = _ints(lit)
        elif coef:
            call = (int(coef), bool(xor))
        elif cmp_name:
            kats["slices"].append({"c": call[0], "xor": call[1], "expect": values[cmp_name]})
    return kats


def one_encode(ref):
    body = _func_body(open(os.path.join(ref, "reedsolomon_test.go")).read(), "TestOneEncode")
    m = re.search(r"New\((\d+),\s*(\d+)", body)
    k, p = int(m.group(1)), int(m.group(2))
    shard_lit = _braced_block(body, body.index("shards := [][]byte") + len("shards := [][]byte") - 1)
    shards = [_ints(s) for s in re.findall(r"\{([^{}]*)\}", shard_lit)]
    expect = {}
    for idx, pos, val in re.findall(r"shards\[(\d+)\]\[(\d+)\]\s*!=\s*(\d+)", body):
        expect.setdefault(int(idx), {})[int(pos)] = int(val)
    parity = {str(i): [expect[i][j] for j in sorted(expect[i])] for i in sorted(expect)}
    return {"k": k, "p": p, "shards": shards, "parity": parity}


def jerasure(ref):
    body = _func_body(open(os.path.join(ref, "reedsolomon_test.go")).read(), "TestBuildMatrixJerasure")
    total = int(re.search(r"totalShards := (\d+)", body).group(1))
    k = int(re.search(r"dataShards := (\d+)", body).group(1))
    lit = _braced_block(body, body.index("refMatrix := matrix") + len("refMatrix := matrix") - 1)
    rows = [_ints(r) for r in re.findall(r"\{([^{}]*)\}", lit)]
    return {"k": k, "total": total, "parity_rows": rows}


def matrix_kats(ref):
    src = open(os.path.join(ref, "matrix_test.go")).read()
    mul = _func_body(src, "TestMatrixMultiply")
    lits = re.findall(r"newMatrixData\(\s*\[\]\[\]byte\{(.*?)\}\)", mul, re.S)
    m1, m2 = ([_ints(r) for r in re.findall(r"\{([^{}]*)\}", l)] for l in lits[:2])
    expect = re.search(r'expect := "([^"]*)"', mul).group(1)
    inv_body = _func_body(src, "TestMatrixInverse")
    cases = []
    for block in re.findall(r"\[\]\[\]byte\{(.*?)\},\s*\n\s*(?://[^\n]*\n\s*)*((?:\"[^\"]*\"\s*\+?\s*)+)", inv_body, re.S):
        rows = [_ints(r) for r in re.findall(r"\{([^{}]*)\}", block[0])]
        text = "".join(re.findall(r'"([^"]*)"', block[1]))
        cases.append({"m": rows, "inverse": text})
    # cases with an empty expected string are the error cases (errNotSquare, errSingular)
    ok = [c for c in cases if c["inverse"]]
    not_square = [c["m"] for c in cases if not c["inverse"] and len(c["m"]) != len(c["m"][0])]
    singular = [c["m"] for c in cases if not c["inverse"] and len(c["m"]) == len(c["m"][0])]
    assert "errSingular" in inv_body and "errNotSquare" in inv_body
    return {"multiply": {"a": m1, "b": m2, "expect": expect}, "inverse": ok,
            "not_square": not_square, "singular": singular}


def addmod(ref, fname, fn, typ):
    body = _func_body(open(os.path.join(ref, fname)).read(), fn)
    pat = r"x:\s*%s\((\d+)\),\s*y:\s*%s\((\d+)\),\s*expected:\s*%s\((\d+)\)" % (typ, typ, typ)
    return [[int(a), int(b), int(c)] for a, b, c in re.findall(pat, body)]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RS_REFERENCE_DIR", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: make_golden.py <reference checkout>")
    out = {
        "tables": galois_tables(ref),
        "galois": galois_kats(ref),
        "one_encode": one_encode(ref),
        "jerasure": jerasure(ref),
        "matrix": matrix_kats(ref),
        "addmod16": addmod(ref, "leopard_test.go", "TestAddMod", "ffe"),
        "addmod8": addmod(ref, "leopard8_test.go", "TestAddMod8", "ffe8"),
    }
    assert len(out["galois"]["slices"]) == 4 and len(out["matrix"]["inverse"]) == 2
    assert len(out["addmod16"]) == 7 and len(out["addmod8"]) == 7
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main()
