"""Builds the in-tree shared library ``libalebgk_b200.so`` for sm_100a.

The library holds the CUDA kernels, the C-ABI of ``include/alebgk.h`` and the
host-side case set-up.  It is compiled with nvcc directly (no JIT cache), so
the ``.so`` sits next to this file and travels with the source tree.

    python -m alebgk4paper_b200.build          # build if sources changed
    python -m alebgk4paper_b200.build --force  # rebuild
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libalebgk_b200.so")

SOURCES = ["step.cu", "march.cu", "body_noalloc.cu", "body_step.cu", "warm.cu", "coeffs_dev.cu", "classes_dev.cu", "setup.cu", "cloud.cu", "checkpoint.cpp", "batch.cpp", "slab.cpp", "api.cpp", "coeffs.cpp", "cases.cpp", "march_plan.cpp", "fields.cpp"]
# The device MLS table builder must round as the host builder (compiled
# without contraction) does.
FILE_FLAGS = {"coeffs_dev.cu": ["-fmad=false"]}
HEADERS = ["ctx.h", "coeffs.h", "cases.h", "march.h", "mbar.cuh", "umma.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the ALE-BGK library needs the CUDA toolkit")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "alebgk.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(ROOT, "_build", "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                     "-I" + os.path.join(ROOT, "include")]
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc()] + common + FILE_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        _run(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lgomp"])
    os.replace(tmp, LIB)
    return LIB


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    if r.stdout.strip() and os.environ.get("ALEBGK_BUILD_VERBOSE"):
        sys.stdout.write(r.stdout)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
