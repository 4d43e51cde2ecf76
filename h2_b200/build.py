"""Build the sm_100a solver library in-tree: h2_b200/libh2g.so.

nvcc compiles the CUDA sources directly for sm_100a (no PTX JIT, no other architectures);
host code is compiled with -ffp-contract=off so the host-side operator tables are evaluated
in the reference's operation order.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libh2g.so")
# (source, extra flags): the model builder is compiled without FMA contraction
SOURCES = [("h2g_solver.cu", []), ("h2g_model.cu", ["-fmad=false"]), ("h2g_noalloc.cu", [])]
DEPS = ["h2g_internal.cuh", "h2g_kernels.cuh", "h2g_sweep.cuh", "h2g_multi.cuh", "h2g_coop.cuh", os.path.join("..", "..", "include", "h2g.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    files = [os.path.join(CSRC, f) for f, _ in SOURCES] + [os.path.join(CSRC, f) for f in DEPS]
    return any(os.path.getmtime(f) > t for f in files)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    log = os.path.join(bdir, "ptxas.log")
    base = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
            "-I", os.path.join(ROOT, "include")]
    objs, text = [], []
    for src, extra in SOURCES:
        obj = os.path.join(bdir, src.replace(".cu", ".o"))
        cmd = base + extra + ["-Xptxas", "-v", "-c", os.path.join(CSRC, src), "-o", obj]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        text.append(" ".join(cmd) + "\n" + proc.stdout + proc.stderr)
        if proc.returncode != 0:
            open(log, "w").write("\n".join(text))
            sys.stderr.write(proc.stdout + proc.stderr)
            raise RuntimeError(f"nvcc failed on {src} ({proc.returncode}); see {log}")
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp"] + objs
    proc = subprocess.run(cmd, capture_output=True, text=True)
    text.append(" ".join(cmd) + "\n" + proc.stdout + proc.stderr)
    open(log, "w").write("\n".join(text))
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc link failed ({proc.returncode}); see {log}")
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print("\n".join(text))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
