"""Times the reference's own GPU path (test infrastructure).

``oracle/_ref/libalebgk_refcuda.so`` holds the reference's CPU set-up and its
CUDA backend ``Solver/CudaBackend.cu``, compiled unmodified for sm_100a by
``make -C oracle refcuda``.  This script builds a case with the reference's
own set-up (TestCases/main.cpp's sequence, via ref_driver.cpp), uploads it
with the reference's cudaUploadCloud, runs ``--warmup`` untimed and
``--steps`` timed cudaStep calls (the body of the reference's GPU time loop,
Solver/Solver.cpp:301-303) and prints one JSON line: ms per step and
particle x velocity updates per second, for the linear MLS the reference
ships and for quadratic MLS.

    python oracle/time_reference_gpu.py --Nx 40 --Nv 10 --warmup 5 --steps 20
"""
from __future__ import annotations

import argparse
import json
import os
import sys

# the repository root, not this folder, so that `oracle` is the package
sys.path[0] = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

from oracle.oracle import RefCase, ref_cuda_library  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="cavity3d")
    ap.add_argument("--Nx", type=int, default=40)
    ap.add_argument("--Nv", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--orders", default="2,1")
    a = ap.parse_args()
    lib = ref_cuda_library()
    if lib is None:
        print(json.dumps({"unavailable": "oracle/_ref/libalebgk_refcuda.so not built"}))
        return
    out = {"case": a.case, "Nx": a.Nx, "Nv": a.Nv, "warmup": a.warmup, "steps": a.steps,
           "impl": "reference Solver/CudaBackend.cu, sm_100a, FP64"}
    for order in [int(o) for o in a.orders.split(",")]:
        r = RefCase(a.case, a.Nx, a.Nv, -1.0, order, fixed_body=True, lib_path=lib)
        ms = r.cuda_run(a.warmup, a.steps)
        updates = r.N * r.Nv ** r.dim
        out[f"mls{order}"] = {"ms_per_step": ms, "updates_per_s": updates / (ms / 1e3),
                              "N": r.N, "velocities": r.Nv ** r.dim}
        del r
    print(json.dumps(out))


if __name__ == "__main__":
    main()
