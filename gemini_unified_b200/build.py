"""Build the CUDA library libgemini_fk.so in-tree for sm_100a.

    python -m gemini_unified_b200.build          # compile if sources changed
    python -m gemini_unified_b200.build --force  # always compile

The parity build of the FK solver (and every other file) is compiled with
--fmad=false so its arithmetic repeats the reference's operation by operation
(the reference is built without FMA contraction); the fast build of the solver
(fk_solver_fast.cu) and the fast inverse FFT (ifft_fast.cu) use FMA contraction.

A build is reused only when the SHA-256 of every source, header, compiler flag
and the compiler's version matches the one recorded beside it, so a library
shipped with newer file times but other sources is rebuilt.

The benchmark's FP64 throughput probe is built as its own library,
libgem_bench_probe.so; the product library does not contain it.
"""
from __future__ import annotations

import concurrent.futures
import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
PROBE_SRC = os.path.join(HERE, "bench_probe", "fp64_probe.cu")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libgemini_fk.so")
PROBE_LIB = os.path.join(OUT_DIR, "libgem_bench_probe.so")
HASH_FILE = os.path.join(OUT_DIR, "build.sha256")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
         "-I" + os.path.join(ROOT, "include")]
# files compiled with FMA contraction; all others repeat the reference's rounding (--fmad=false)
FMAD_TRUE = {"fk_solver_fast.cu", "ifft_fast.cu", "legendre_fast.cu", "proposer.cu"}


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _inputs():
    return sorted(sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")) + [PROBE_SRC])


def _nvcc_version() -> str:
    try:
        return subprocess.run([NVCC, "--version"], capture_output=True, text=True).stdout
    except OSError:
        return "nvcc unavailable"


def source_hash() -> str:
    h = hashlib.sha256()
    for f in _inputs():
        h.update(os.path.relpath(f, ROOT).encode())
        with open(f, "rb") as fh:
            h.update(hashlib.sha256(fh.read()).digest())
    h.update(repr((ARCH, FLAGS, sorted(FMAD_TRUE))).encode())
    h.update(_nvcc_version().encode())
    return h.hexdigest()


def _stale(digest: str) -> bool:
    if not (os.path.exists(LIB) and os.path.exists(PROBE_LIB) and os.path.exists(HASH_FILE)):
        return True
    with open(HASH_FILE) as fh:
        return fh.read().strip() != digest


def build(force: bool = False, verbose: bool = False) -> str:
    digest = source_hash()
    if not force and not _stale(digest):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    if os.path.exists(HASH_FILE):
        os.unlink(HASH_FILE)

    def compile_one(src):
        obj = os.path.join(OUT_DIR, os.path.basename(src)[:-3] + ".o")
        fmad = "--fmad=true" if os.path.basename(src) in FMAD_TRUE else "--fmad=false"
        cmd = [NVCC, *ARCH, *FLAGS, fmad, "-c", src, "-o", obj]
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units are independent: compile them in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as pool:
        results = list(pool.map(compile_one, sources() + [PROBE_SRC]))
    objs, logs, probe_obj = [], [], None
    for src, obj, r in results:
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stdout + r.stderr))
        if src == PROBE_SRC:
            probe_obj = obj
        else:
            objs.append(obj)
    for out, ins in ((LIB, objs), (PROBE_LIB, [probe_obj])):
        tmp = out + ".tmp"
        r = subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *ins, "-lcudart"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link of %s failed:\n%s" % (os.path.basename(out), r.stdout + r.stderr))
        os.replace(tmp, out)
    with open(os.path.join(OUT_DIR, "ptxas.log"), "w") as fh:
        fh.write("\n".join(logs))
    with open(HASH_FILE, "w") as fh:
        fh.write(digest + "\n")
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
