"""Checks the reference-side shim ``alebgk4paper_b200/shim/cuda_backend_shim.cpp``
(test infrastructure, run where the reference sources are present).

1. The shim is compiled against the reference's own headers and this
   project's ``include/alebgk.h``.
2. The reference's ``Solver/Solver.cpp`` is compiled with ``ALEBGK_WITH_CUDA``
   (the build in which it calls the CUDA backend, ``Solver.cpp:67-89``).
3. Every CUDA-backend symbol the solver object leaves undefined must be
   defined by the shim object, with the same C++ signature.

Exit status 0: the shim covers the solver; 1: it does not (the missing
symbols are printed); 77: the reference sources or g++ are absent.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = os.environ.get("ALEBGK_REF", "/root/reference")


SHIM = os.path.join(ROOT, "alebgk4paper_b200", "shim", "cuda_backend_shim.cpp")


def symbols(obj: str, defined: bool) -> set[str]:
    flag = "--defined-only" if defined else "--undefined-only"
    out = subprocess.run(["nm", "-C", flag, obj], capture_output=True, text=True, check=True)
    syms = set()
    for line in out.stdout.splitlines():
        parts = line.split(None, 2 if defined else 1)
        name = parts[-1].strip()
        if name.startswith("cuda"):
            syms.add(name)
    return syms


def main() -> int:
    solver = os.path.join(REF, "Solver", "Solver.cpp")
    if not os.path.exists(solver) or not shutil.which("g++") or not shutil.which("nm"):
        print("reference sources or toolchain absent")
        return 77
    inc = [f"-I{os.path.join(REF, d)}" for d in sorted(os.listdir(REF))
           if os.path.isdir(os.path.join(REF, d))]
    with tempfile.TemporaryDirectory() as tmp:
        shim = SHIM
        base = ["g++", "-std=c++17", "-O0", "-fopenmp", "-w"] + inc
        subprocess.run(base + ["-DALEBGK_WITH_CUDA", "-c", solver, "-o",
                               os.path.join(tmp, "solver.o")], check=True)
        subprocess.run(base + [f"-I{os.path.join(ROOT, 'include')}", "-c", shim, "-o",
                               os.path.join(tmp, "shim.o")], check=True)
        need = symbols(os.path.join(tmp, "solver.o"), defined=False)
        have = symbols(os.path.join(tmp, "shim.o"), defined=True)
    missing = sorted(need - have)
    print(f"{len(need)} CUDA-backend symbols referenced by Solver.cpp; "
          f"{len(need) - len(missing)} defined by the shim")
    for m in missing:
        print("missing:", m)
    return 1 if missing or not need else 0


if __name__ == "__main__":
    sys.exit(main())
