"""The generated XOR-network kernel (GF(2^8) variant 7) on the device:
bit-exact with the oracle when chosen by the tuner rather than forced, i.e.
on the first uses of a matrix (a table kernel runs; the second use queues
the network's compile in the background) and after the compile; in every
mode; with a sub-chunk tail; for decode matrices; inside a captured batch
graph."""
import numpy as np
import pytest
import torch

import oracle as O
import reedsolomon_b200 as rs

pytestmark = pytest.mark.gpu

lib = rs.lib()
needs_nvrtc = pytest.mark.skipif(not lib.rsgpu_xornet_available(), reason="NVRTC not loadable")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


class tuned:
    """Records variant 7 for the given (n_in, n_out, size, mode) geometries."""

    def __init__(self, *geos):
        self.geos = geos

    def __enter__(self):
        for ni, no, size, mode in self.geos:
            assert lib.rsgpu_record_variant(ni, no, size, mode, 7) == 0

    def __exit__(self, *exc):
        for ni, no, size, mode in self.geos:
            lib.rsgpu_record_variant(ni, no, size, mode, -1)


def stripe(k, p, size, seed):
    data = O.seeded_shards(seed, k, size)
    want = data + [np.zeros(size, np.uint8) for _ in range(p)]
    O.rs_encode(k, p, want)
    return data, want


@needs_nvrtc
@pytest.mark.parametrize("k,p,size", [(6, 3, 65536 + 3 * 1024 + 7), (11, 5, 1 << 20), (4, 2, 1024)])
def test_tuned_encode_first_sight_and_compiled(k, p, size):
    data, want = stripe(k, p, size, seed=k * 100 + p)
    enc = rs.New(k, p)
    with tuned((k, p, size, 0), (k, p, size, 2)):
        for rnd in range(3):   # first sight and second use (table kernel), then the compiled network
            sh = [dev(d) for d in data] + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
            enc.Encode(sh)
            for i in range(k, k + p):
                assert np.array_equal(host(sh[i]), want[i]), (rnd, i)
            assert enc.Verify(sh)
            sh[k + p - 1][size // 2] ^= 1
            assert not enc.Verify(sh)
            if rnd == 1:
                assert lib.rsgpu_xornet_sync() >= 1


@needs_nvrtc
def test_tuned_reconstruct_decode_matrices():
    k, p, size = 8, 4, 262144 + 64
    data, want = stripe(k, p, size, seed=31)
    enc = rs.New(k, p)
    patterns = [(0, 9), (1, 2, 3, 11), (7,), (4, 8, 10)]
    geos = [(k, n, size, 0) for n in (1, 2, 3, 4)]
    with tuned(*geos):
        for rnd in range(3):
            for lost in patterns:
                sh = [None if i in lost else dev(want[i]) for i in range(k + p)]
                enc.Reconstruct(sh)
                for i in lost:
                    assert np.array_equal(host(sh[i]), want[i]), (rnd, lost, i)
            lib.rsgpu_xornet_sync()


@needs_nvrtc
def test_xor_mode_accumulates_over_input_tiles():
    """k > 32 splits the inputs: the first tile writes, later tiles XOR."""
    k, p, size = 40, 3, 8192
    data, want = stripe(k, p, size, seed=40)
    enc = rs.New(k, p)
    with tuned((32, p, size, 0), (8, p, size, 1)):
        for rnd in range(3):
            sh = [dev(d) for d in data] + [torch.full((size,), 0x5A, dtype=torch.uint8, device="cuda")
                                           for _ in range(p)]
            enc.Encode(sh)
            for i in range(k, k + p):
                assert np.array_equal(host(sh[i]), want[i]), (rnd, i)
            lib.rsgpu_xornet_sync()


@needs_nvrtc
def test_batch_graph_capture_with_tuned_network():
    """A captured batch graph runs the table kernel for a network that was
    never loaded, and the network itself once an uncaptured launch loaded it."""
    k, p, size, n = 5, 3, 8192, 6
    stripes = [stripe(k, p, size, seed=500 + s) for s in range(n)]

    def run(mode):
        b = rs.Batch()
        outs = []
        for data, _ in stripes:
            sh = [dev(d) for d in data] + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
            b.add_encode(k, p, sh)
            outs.append(sh)
        b.run(mode)
        for (data, want), sh in zip(stripes, outs):
            for i in range(k, k + p):
                assert np.array_equal(host(sh[i]), want[i]), (mode, i)

    with tuned((k, p, size, 0)):
        run("graph")           # compile queued; capture used the table kernel
        lib.rsgpu_xornet_sync()
        run("per_stripe")      # loads the compiled network
        run("graph")           # captured with the network


@needs_nvrtc
@pytest.mark.parametrize("skew", [1, 8, 16])
def test_forced_network_with_unaligned_shards(skew):
    """Shards off the 16-byte grid (skew 1, 8) cannot use the vector network:
    the table kernels take over.  On the grid (skew 16) the network covers
    the whole 1 KiB chunks and a table kernel the 5-byte tail.  Bytes around
    every shard stay untouched."""
    k, p, size = 6, 3, (256 << 10) + 5
    data, want = stripe(k, p, size, seed=600 + skew)
    pitch = (size + 64 + 15) // 16 * 16
    buf = torch.full(((k + p) * pitch,), 0xA5, dtype=torch.uint8, device="cuda")
    sh = [buf[i * pitch + skew: i * pitch + skew + size] for i in range(k + p)]
    for i in range(k):
        sh[i].copy_(dev(data[i]))
    assert lib.rsgpu_force_variant(7) == 0
    try:
        enc = rs.New(k, p)
        enc.Encode(sh)
        for i in range(k, k + p):
            assert np.array_equal(host(sh[i]), want[i]), i
        assert enc.Verify(sh)
    finally:
        lib.rsgpu_force_variant(-1)
    h = host(buf).reshape(k + p, pitch)
    assert (h[:, :skew] == 0xA5).all() and (h[:, skew + size:] == 0xA5).all()


@needs_nvrtc
def test_forced_network_wide_tile_1mib():
    """32 x 16 tile (256-thread kernel, smaller factoring groups) at 1 MiB,
    where launches use fewer warps per CTA to cover every SM."""
    k, p, size = 32, 16, 1 << 20
    data, want = stripe(k, p, size, seed=3216)
    assert lib.rsgpu_force_variant(7) == 0
    try:
        enc = rs.New(k, p)
        sh = [dev(d) for d in data] + [torch.zeros(size, dtype=torch.uint8, device="cuda") for _ in range(p)]
        enc.Encode(sh)
        for i in range(k, k + p):
            assert np.array_equal(host(sh[i]), want[i]), i
        assert enc.Verify(sh)
        sh[k + 7][size - 1] ^= 2
        assert not enc.Verify(sh)
    finally:
        lib.rsgpu_force_variant(-1)


def test_python_autotune_helper():
    """rs.autotune times every variant (the XOR network included when NVRTC
    is present) and records the fastest; record_variant(None) removes it."""
    best, ms = rs.autotune(10, 4, 1 << 20)
    assert best in ms and all(v > 0 for v in ms.values())
    assert (rs.VARIANT_XORNET in ms) == bool(lib.rsgpu_xornet_available())
    best_v, ms_v = rs.autotune(10, 4, 1 << 20, mode="verify", reps=2)
    assert best_v in ms_v
    rs.record_variant(10, 4, 1 << 20, None)
    rs.record_variant(10, 4, 1 << 20, None, mode="verify")


@needs_nvrtc
def test_disk_cached_kernels_load_and_match(tmp_path):
    """With RSGPU_KERNEL_CACHE set, one process compiles and stores the
    kernel, a second loads the stored cubin without compiling; both encode
    bit-exactly."""
    import os
    import subprocess
    import sys
    code = (
        "import numpy as np, torch, oracle as O, reedsolomon_b200 as rs\n"
        "k, p, S = 7, 3, 1 << 20\n"
        "data = O.seeded_shards(4242, k, S); want = data + [np.zeros(S, np.uint8) for _ in range(p)]\n"
        "O.rs_encode(k, p, want)\n"
        "rs.force_variant(7)\n"
        "sh = [torch.from_numpy(d).cuda() for d in data] + [torch.zeros(S, dtype=torch.uint8, device='cuda') for _ in range(p)]\n"
        "rs.New(k, p).Encode(sh)\n"
        "assert all(np.array_equal(sh[i].cpu().numpy(), want[i]) for i in range(k, k + p))\n"
        "print('files', len(__import__('os').listdir(__import__('os').environ['RSGPU_KERNEL_CACHE'])))\n")
    env = dict(os.environ, RSGPU_KERNEL_CACHE=str(tmp_path / "kc"))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env["PYTHONPATH"] = root + os.pathsep + env.get("PYTHONPATH", "")
    outs, stamps = [], []
    for _ in range(2):
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
        outs.append(r.stdout.strip())
        (f,) = list((tmp_path / "kc").iterdir())
        stamps.append(f.stat().st_mtime_ns)
    assert outs[0] == outs[1] == "files 1"
    assert stamps[0] == stamps[1]   # the second process loaded the file, it did not rewrite it
