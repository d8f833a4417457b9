"""The generated XOR-network schedule (variant 7 of the GF(2^8) kernel),
checked on the CPU: librsgpu emits the same schedule the CUDA kernel runs as
a plain C function (rs_xornet_host), one per mode; gcc compiles it and its
outputs in the write / xor / verify modes must equal the oracle's
codeSomeShards over random and reference encoding matrices."""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")


WRITE, XOR, VERIFY = 0, 1, 2


def source(coef, mode, host, group=0):
    lib = rs.lib()
    coef = np.ascontiguousarray(coef, np.uint8)
    no, ni = coef.shape
    n = lib.rsgpu_xornet_source(coef.ctypes.data, ni, no, mode, group, host, None, 0)
    assert n > 0
    buf = ctypes.create_string_buffer(n + 1)
    assert lib.rsgpu_xornet_source(coef.ctypes.data, ni, no, mode, group, host, buf, n + 1) == n
    return buf.value.decode()


def host_kernel(coef, mode, tmp_path, group=0):
    c = tmp_path / ("xn%d_%d.c" % (mode, group))
    so = tmp_path / ("xn%d_%d.so" % (mode, group))
    c.write_text(source(coef, mode, 1, group))
    r = subprocess.run(["gcc", "-O0", "-shared", "-fPIC", "-o", str(so), str(c)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[:2000]
    return ctypes.CDLL(str(so))


def run(h, ins, outs):
    n = ins[0].size
    assert n % 1024 == 0
    ip = (ctypes.c_void_p * len(ins))(*[a.ctypes.data for a in ins])
    op = (ctypes.c_void_p * len(outs))(*[a.ctypes.data for a in outs])
    flag = ctypes.c_int(0)
    h.rs_xornet_host(ip, op, ctypes.c_longlong(n // 1024), ctypes.byref(flag))
    return flag.value


def reference_parity(k, p):
    _, m = O.build_matrix("default", k, k + p)
    return m[k:]


CASES = [("rs10x4", 10, 4), ("rand1x1", 1, 1), ("rand3x7", 3, 7), ("rand32x16", 32, 16),
         ("rand17x3", 17, 3), ("rand2x16", 2, 16), ("rs6x3", 6, 3), ("rand32x8", 32, 8)]


GROUP_CASES = [(n, i, o, 0) for n, i, o in CASES] + \
    [("rs10x4", 10, 4, 1), ("rs10x4", 10, 4, 2), ("rand3x7", 3, 7, 1), ("rand32x8", 32, 8, 1)]


@pytest.mark.parametrize("name,ni,no,group", GROUP_CASES)
def test_generated_schedule_matches_oracle(name, ni, no, group, tmp_path):
    rng = np.random.default_rng(ni * 131 + no)
    coef = reference_parity(ni, no) if name.startswith("rs") else rng.integers(0, 256, (no, ni), dtype=np.uint8)
    n = 3 * 1024
    ins = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(ni)]
    want = [np.zeros(n, np.uint8) for _ in range(no)]
    O.code_some_shards(coef, ins, want)
    h = host_kernel(coef, WRITE, tmp_path, group)
    outs = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(no)]   # overwritten in write mode
    run(h, ins, outs)
    for j in range(no):
        assert np.array_equal(outs[j], want[j]), (name, j)
    h = host_kernel(coef, XOR, tmp_path, group)
    base = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(no)]
    acc = [b.copy() for b in base]
    run(h, ins, acc)
    for j in range(no):
        assert np.array_equal(acc[j], base[j] ^ want[j]), (name, j)
    h = host_kernel(coef, VERIFY, tmp_path, group)
    assert run(h, ins, [w.copy() for w in want]) == 0
    bad = [w.copy() for w in want]
    bad[no - 1][n - 1] ^= 0x40
    assert run(h, ins, bad) == 1
    bad = [w.copy() for w in want]
    bad[0][0] ^= 0x01
    assert run(h, ins, bad) == 1


def test_zero_and_identity_coefficients(tmp_path):
    """Rows of zeros produce zero planes; an identity row copies its input."""
    coef = np.zeros((3, 4), np.uint8)
    coef[1, 2] = 1
    coef[2, :] = [1, 1, 0, 0]
    h = host_kernel(coef, WRITE, tmp_path)
    rng = np.random.default_rng(9)
    ins = [rng.integers(0, 256, 1024, dtype=np.uint8) for _ in range(4)]
    outs = [np.full(1024, 0xFF, np.uint8) for _ in range(3)]
    run(h, ins, outs)
    assert not outs[0].any()
    assert np.array_equal(outs[1], ins[2])
    assert np.array_equal(outs[2], ins[0] ^ ins[1])


def test_source_is_deterministic_and_bounded():
    coef = reference_parity(10, 4)
    a, b = source(coef, WRITE, 0), source(coef, WRITE, 0)
    assert a == b
    assert "rs_xornet" in a and "__launch_bounds__" in a
    assert source(coef, VERIFY, 0) != a
    lib = rs.lib()
    c = np.ascontiguousarray(coef)
    assert lib.rsgpu_xornet_source(c.ctypes.data, 33, 4, 0, 0, 0, None, 0) < 0     # more than 32 inputs
    assert lib.rsgpu_xornet_source(c.ctypes.data, 10, 17, 0, 0, 0, None, 0) < 0    # more than 16 outputs
    assert lib.rsgpu_xornet_source(c.ctypes.data, 10, 4, 3, 0, 0, None, 0) < 0     # no such mode
    assert lib.rsgpu_xornet_source(c.ctypes.data, 10, 4, 0, -1, 0, None, 0) < 0    # bad group
    small = ctypes.create_string_buffer(16)
    n = lib.rsgpu_xornet_source(c.ctypes.data, 10, 4, 0, 0, 0, small, 16)
    assert n == len(a) and len(small.value) == 15


def _nvrtc():
    try:
        return ctypes.CDLL("libnvrtc.so.12")
    except OSError:
        return None


@pytest.mark.skipif(_nvrtc() is None, reason="libnvrtc.so.12 not loadable")
@pytest.mark.parametrize("ni,no,mode,group", [(10, 4, WRITE, 0), (10, 4, VERIFY, 0), (10, 4, XOR, 0),
                                              (17, 3, WRITE, 2), (32, 16, WRITE, 1), (5, 9, VERIFY, 0)])
def test_generated_cuda_compiles_for_sm100a(ni, no, mode, group):
    """The device form of the same schedule goes through NVRTC for sm_100a
    (no GPU needed) and exports the kernel the library loads."""
    nv = _nvrtc()
    rng = np.random.default_rng(ni + 7 * no)
    coef = reference_parity(ni, no) if (ni, no) == (10, 4) else rng.integers(0, 256, (no, ni), dtype=np.uint8)
    src = source(coef, mode, 0, group).encode()
    prog = ctypes.c_void_p()
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), src, b"rs_xornet.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"--std=c++17", b"-default-device"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    n = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value)
    nv.nvrtcGetProgramLog(prog, log)
    assert rc == 0, log.value.decode()[:2000]
    size = ctypes.c_size_t()
    assert nv.nvrtcGetCUBINSize(prog, ctypes.byref(size)) == 0 and size.value > 0
    nv.nvrtcDestroyProgram(ctypes.byref(prog))


def test_nvrtc_switch_off_disables_variant_7():
    """RSGPU_NVRTC=off: no XOR-network kernels; the library still loads and
    reports the variant unavailable (the table kernels then run)."""
    import os
    import sys
    code = ("import reedsolomon_b200 as rs; l = rs.lib(); "
            "print(l.rsgpu_xornet_available(), l.rsgpu_xornet_sync())")
    env = dict(os.environ, RSGPU_NVRTC="off")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split() == ["0", "0"]
    env["RSGPU_NVRTC"] = ""
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.split()[0] == ("1" if _nvrtc() else "0")


def test_record_and_force_variant_arguments():
    """The tuning records need no device: bad geometries, modes and variants
    are refused; a recorded choice can be removed again."""
    lib = rs.lib()
    n = lib.rsgpu_num_variants()
    assert n == 9
    assert lib.rsgpu_record_variant(10, 4, 1 << 20, 0, 7) == 0
    assert lib.rsgpu_record_variant(10, 4, 1 << 20, 0, -1) == 0
    for args in [(0, 4, 1 << 20, 0, 7), (33, 4, 1 << 20, 0, 7), (10, 17, 1 << 20, 0, 7), (10, 4, 0, 0, 7),
                 (10, 4, 1 << 20, 3, 7), (10, 4, 1 << 20, 0, n), (10, 4, 1 << 20, 0, -2)]:
        assert lib.rsgpu_record_variant(*args) < 0, args
    assert lib.rsgpu_force_variant(n) < 0
    assert lib.rsgpu_force_variant(-1) == 0


def test_python_tuning_helpers_without_device():
    assert rs.generated_kernels_available() == bool(_nvrtc())
    rs.record_variant(10, 4, 1 << 20, rs.VARIANT_XORNET)
    rs.record_variant(10, 4, 1 << 20, None)
    rs.record_variant(10, 4, 1 << 20, 3, mode="verify")
    rs.record_variant(10, 4, 1 << 20, None, mode="verify")
    rs.force_variant(6)
    rs.force_variant(None)
    with pytest.raises(rs.RSError):
        rs.force_variant(99)
    assert rs.wait_generated_kernels() >= 0


@pytest.mark.skipif(_nvrtc() is None, reason="libnvrtc.so.12 not loadable")
def test_prepare_kernels_without_device():
    """PrepareKernels compiles the Encode/Verify networks of a host-only
    encoder: one write and one compare kernel for k <= 32; for k = 40,
    p = 20 the write kernel of the first input tile and the xor kernels of
    the second, for both output tiles (verify composes write kernels)."""
    before = rs.wait_generated_kernels()
    assert rs.New(10, 4, rs.HostOnly()).PrepareKernels() == 2
    assert rs.New(40, 20, rs.HostOnly()).PrepareKernels() == 4
    assert rs.New(10, 4, rs.HostOnly(), rs.WithLeopardGF16()).PrepareKernels() == 0
    assert rs.wait_generated_kernels() >= before + 6
    assert rs.New(10, 4, rs.HostOnly()).PrepareKernels() == 2   # cached: no new compile


def _network_xors(src):
    body = src[src.index("for (; c < XN_N"):]
    return sum(line.count("^") for line in body.split("\n")
               if (line.startswith("o") and "^=" in line) or line.startswith("const u32 t"))


def test_factoring_keeps_the_network_small():
    """The generated RS(10,4) network needs 632 two-input XORs after pair
    factoring, about half of the 1224 single-bit terms of its bit matrix; a
    generator change that loses the factoring shows up here before it shows
    up as a slower kernel."""
    coef = reference_parity(10, 4)
    terms = sum(bin(O.gal_mul(int(coef[j][i]), 1 << a)).count("1")
                for j in range(4) for i in range(10) for a in range(8))
    assert terms == 1224
    assert _network_xors(source(coef, WRITE, 0)) <= 660


@pytest.mark.skipif(_nvrtc() is None, reason="libnvrtc.so.12 not loadable")
@pytest.mark.parametrize("ni,no,mode", [(1, 1, WRITE), (32, 1, VERIFY), (1, 16, XOR), (32, 16, VERIFY), (2, 7, WRITE)])
def test_corner_tiles_compile(ni, no, mode):
    """Extreme tile shapes, each in the group size the library tries first,
    go through NVRTC for sm_100a."""
    nv = _nvrtc()
    coef = np.random.default_rng(ni * 17 + no).integers(0, 256, (no, ni), dtype=np.uint8)
    src = source(coef, mode, 0).encode()
    prog = ctypes.c_void_p()
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), src, b"rs_xornet.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"--std=c++17", b"-default-device"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    assert rc == 0
