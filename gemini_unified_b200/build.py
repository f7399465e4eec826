"""Build the CUDA library libgemini_fk.so in-tree for sm_100a.

    python -m gemini_unified_b200.build          # compile if sources changed
    python -m gemini_unified_b200.build --force  # always compile

The parity build of the FK solver (and every other file) is compiled with
--fmad=false so its arithmetic repeats the reference's operation by operation
(the reference is built without FMA contraction); the fast build of the solver
(fk_solver_fast.cu) and the fast inverse FFT (ifft_fast.cu) use FMA contraction.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libgemini_fk.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
         "-I" + os.path.join(ROOT, "include")]
# files compiled with FMA contraction; all others repeat the reference's rounding (--fmad=false)
FMAD_TRUE = {"fk_solver_fast.cu", "ifft_fast.cu", "legendre_fast.cu", "proposer.cu"}


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(OUT_DIR, os.path.basename(src)[:-3] + ".o")
        fmad = "--fmad=true" if os.path.basename(src) in FMAD_TRUE else "--fmad=false"
        cmd = [NVCC, *ARCH, *FLAGS, fmad, "-c", src, "-o", obj]
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units are independent: compile them in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as pool:
        results = list(pool.map(compile_one, sources()))
    objs, logs = [], []
    for src, obj, r in results:
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stdout + r.stderr))
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    with open(os.path.join(OUT_DIR, "ptxas.log"), "w") as fh:
        fh.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
