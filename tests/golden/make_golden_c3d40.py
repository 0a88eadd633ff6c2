"""Generates the full-size cavity3d fixture from the reference itself.

cavity3d, Nx = 40 (64 000 particles), Nv = 10 (1 000 velocities), quadratic
MLS, the case's default dt, stepped by the reference's own CPU code
(``oracle/_ref``, compiled unmodified by ``oracle/Makefile``) through
``oracle/ref_driver.cpp`` with the reference's step order
(Solver/Solver.cpp:632-705).  The full distribution is 512 MB, so the
fixture keeps, at steps 1, 10 and 50:

* the moment fields rho, ux, uy, uz, T of every particle,
* the row sums sum_k g and sum_k |g| of every particle,
* 256 seeded full rows of g (walls, corners and interior alike),

plus the transport-flag and moodCheck counts and the total mass of every
step.  About fifteen minutes on eight cores::

    make -C oracle ref && python tests/golden/make_golden_c3d40.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import RefCase  # noqa: E402

CHECKPOINTS = (1, 10, 50)
NROWS = 256
FIXTURE = "step_c3d_n40_v10_q_s1_s10_s50.npz"
SEED = 40


def main():
    r = RefCase("cavity3d", 40, 10, -1.0, 2, fixed_body=True)
    r.set_threads(r.max_threads())
    rows = np.sort(np.random.default_rng(SEED).choice(r.N, NROWS, replace=False))
    out = dict(case="cavity3d", Nx=40, Nv=10, order=2, rows=rows)
    flags, mass = [], []
    for step in range(1, max(CHECKPOINTS) + 1):
        t0 = time.time()
        st = r.step(1)
        flags.append([st["transport_flags"], st["mood_fail"]])
        mass.append(r.sum_mass())
        print(f"step {step}: {time.time() - t0:.1f} s, flags {flags[-1]}", flush=True)
        if step in CHECKPOINTS:
            g = r.g()
            out[f"macro_s{step}"] = r.macro()[:, :5].copy()
            out[f"gsum_s{step}"] = g.sum(axis=1)
            out[f"gabs_s{step}"] = np.abs(g).sum(axis=1)
            out[f"g_s{step}"] = g[rows].copy()
            del g
    out["flags"] = np.array(flags)
    out["mass"] = np.array(mass)
    np.savez_compressed(os.path.join(HERE, FIXTURE), **out)
    print("written", os.path.join(HERE, FIXTURE))


if __name__ == "__main__":
    main()
