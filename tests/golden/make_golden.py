"""Generates the golden fixtures in this folder from the reference itself.

The reference ships no tests or golden vectors, so every fixture here is the
output of the reference's own CPU code (compiled unmodified by
``oracle/Makefile`` into ``oracle/_ref/``), run through ``oracle/ref_driver.cpp``
with the reference's set-up and step order.  Re-run after rebuilding
``oracle/_ref``::

    make -C oracle ref && python tests/golden/make_golden.py [tag ...]

With tags, only the step fixtures of those tags are written.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import RefCase  # noqa: E402

# (case, Nx, Nv, mls_order, fixed body)
SETUPS = [
    ("cavity2d", 12, 8, 2, True),
    ("cavity3d", 6, 4, 2, True),
    ("cavity2d-square", 24, 8, 2, True),
    ("cavity2d-circle", 20, 8, 2, True),
    ("cavity3d-sphere", 12, 4, 2, True),
    ("cavity3d-cube", 12, 4, 2, True),
]

# (tag, case, Nx, Nv, mls_order, steps, keep full g)
STEPS = [
    ("c2d_n8_v8_q_s5", "cavity2d", 8, 8, 2, 5, True),
    ("c2d_n20_v16_q_s20", "cavity2d", 20, 16, 2, 20, False),
    ("c2d_n20_v16_l_s20", "cavity2d", 20, 16, 1, 20, False),
    ("c3d_n6_v4_q_s3", "cavity3d", 6, 4, 2, 3, True),
    ("c3d_n10_v6_q_s3", "cavity3d", 10, 6, 2, 3, False),
    ("c3d_n9_v5_q_s3", "cavity3d", 9, 5, 2, 3, False),
    ("cube_n12_v4_q_s2", "cavity3d-cube", 12, 4, 2, 2, False),
    ("square_n24_v8_q_s4", "cavity2d-square", 24, 8, 2, 4, False),
]

# Long runs, held to the FP64 contract on the moment fields (1e-6 relative)
# rather than to rounding: the plain cavity2d (Nx 20, Nv 16, quadratic,
# default dt) over its full 500 steps, in which the quadratic scheme turns
# unstable and amplifies rounding differences.
LONG_STEPS = [
    ("c2d_n20_v16_q_s500", "cavity2d", 20, 16, 2, 500, False),
]

# Free-body runs: (tag, case, Nx, Nv), BODY_STEPS steps each.
BODY_RUNS = [
    ("cube_n12_v4_free", "cavity3d-cube", 12, 4),
    ("square_n24_v8_free", "cavity2d-square", 24, 8),
]
BODY_STEPS = 8
# A long free-body run: the cube of cavity3d-cube (Nx 12, Nv 4) moves three
# to four lattice steps and turns by 110 degrees in 2000 steps, and the cloud
# management changes the particle set on most steps after step 254.  Kept:
# the particle count after every step and the body state every 10 steps.
LONG_BODY = ("cube_n12_v4_free_s2000", "cavity3d-cube", 12, 4, 2000, 10)


def write_long_body(tag, case, Nx, Nv, steps, every):
    r = RefCase(case, Nx, Nv, -1.0, 2, fixed_body=False)
    b0 = r.bodies().copy()
    hist, counts = [], []
    for k in range(1, steps + 1):
        r.step(1)
        counts.append(r.N)
        if k % every == 0:
            hist.append(r.bodies().copy())
    np.savez_compressed(os.path.join(HERE, f"body_{tag}.npz"), bodies_before=b0,
                        bodies=np.array(hist), N=np.array(counts), every=every)


def nbr_hash(nbr: np.ndarray, nnb: np.ndarray) -> np.ndarray:
    """Order-sensitive per-particle hash of the neighbour list."""
    out = np.zeros(len(nnb), np.int64)
    for i, n in enumerate(nnb):
        h = 1469598103934665603
        for j in nbr[i, :n]:
            h = ((h ^ int(j)) * 1099511628211) & 0x7FFFFFFFFFFFFFFF
        out[i] = h
    return out


def write_step(tag, case, Nx, Nv, order, steps, full):
    r = RefCase(case, Nx, Nv, -1.0, order, fixed_body=True)
    flags = []
    for _ in range(steps):
        st = r.step(1)
        flags.append([st["transport_flags"], st["mood_fail"]])
    g = r.g()
    d = dict(case=case, Nx=Nx, Nv=Nv, order=order, steps=steps, macro=r.macro(),
             gsum=g.sum(axis=1), gabs=np.abs(g).sum(axis=1), flags=np.array(flags),
             mass=r.sum_mass())
    if full:
        d["g"] = g
    np.savez_compressed(os.path.join(HERE, f"step_{tag}.npz"), **d)


def main(only=None):
    if only:
        for tag, case, Nx, Nv, order, steps, full in STEPS + LONG_STEPS:
            if tag in only:
                write_step(tag, case, Nx, Nv, order, steps, full)
        if LONG_BODY[0] in only:
            write_long_body(*LONG_BODY)
        return
    for case, Nx, Nv, order, fixed in SETUPS:
        r = RefCase(case, Nx, Nv, -1.0, order, fixed_body=fixed)
        c = r.cloud()
        np.savez_compressed(
            os.path.join(HERE, f"setup_{case}_n{Nx}_v{Nv}.npz"),
            xyz=c["xyz"], wall=c["wall"], boundary=c["boundary"], body_id=c["body_id"],
            nnb=c["nnb"], nbr_hash=nbr_hash(c["nbr"], c["nnb"]), g0=r.g()[:4],
            params=np.array([r.params[k] for k in ("dt", "tau", "R", "dx", "radius", "dv",
                                                   "vmin", "rho0", "Tw")]))
    for tag, case, Nx, Nv, order, steps, full in STEPS + LONG_STEPS:
        write_step(tag, case, Nx, Nv, order, steps, full)
    # Free bodies: the reference's moving-body path (fluid step, then
    # moveRigidBodies, RigidBody/BodyDynamics.cpp:143-711, then its cloud
    # management) -> body state and particle count after every step.
    for tag, case, Nx, Nv in BODY_RUNS:
        r = RefCase(case, Nx, Nv, -1.0, 2, fixed_body=False)
        b0 = r.bodies().copy()
        hist, counts = [], []
        for _ in range(BODY_STEPS):
            r.step(1)
            hist.append(r.bodies().copy())
            counts.append(r.N)
        np.savez_compressed(os.path.join(HERE, f"body_{tag}.npz"), bodies_before=b0,
                            bodies=np.array(hist), N=np.array(counts))
    write_long_body(*LONG_BODY)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1:])
