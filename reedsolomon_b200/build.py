"""Build librsgpu.so in-tree for sm_100a.

    python -m reedsolomon_b200.build            # incremental
    python -m reedsolomon_b200.build --force    # rebuild everything
    python -m reedsolomon_b200.build --ptxas-v  # print register / smem usage

Every .cu/.cpp under csrc/ is compiled by nvcc with
-gencode arch=compute_100a,code=sm_100a and linked against the static CUDA
runtime, so the shared object carries no dependency on a particular
libcudart and can be loaded next to PyTorch's runtime.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librsgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
GEN = os.path.join(BUILD, "gen")  # generated headers (gen_rt_dispatch.py)

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", INCLUDE, "-I", CSRC, "-I", GEN]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _generate():
    """Writes the generated headers (rewritten only when their text changes)."""
    from reedsolomon_b200 import gen_rt_dispatch
    gen_rt_dispatch.write(os.path.join(GEN, "gf8_rt_dispatch.inc"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(GEN, f) for f in os.listdir(GEN) if f.endswith(".inc")]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def _compile(src, obj, ptxas_v):
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["--expt-relaxed-constexpr"]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stdout + r.stderr))
    return r.stdout + r.stderr


def build(force=False, ptxas_v=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    _generate()
    hdr = _headers_mtime()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        stale = force or ptxas_v or not os.path.exists(obj) or \
            os.path.getmtime(obj) < max(os.path.getmtime(src), hdr)
        if stale:
            jobs.append((src, obj))
    logs = []
    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, ptxas_v) for s, o in jobs]
            for f in futs:
                logs.append(f.result())
    need_link = jobs or not os.path.exists(LIB) or \
        os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)
    if need_link:
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stdout + r.stderr))
    if verbose or ptxas_v:
        for l in logs:
            if l.strip():
                print(l)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, ptxas_v="--ptxas-v" in sys.argv, verbose=True))
