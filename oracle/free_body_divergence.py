"""Test infrastructure: where the free-cube run of cavity3d-cube (Nx 40, Nv 10)
diverges, on this library and on the compiled reference from the same state.

Runs the FP64 device step (fluid step, Heun body step, cloud management) to
step S0, writes the state as a restart file in the reference's layout
(Core/Checkpoint.hpp), steps the device on while printing the density range
and the cube's velocity per step, then restores the file into the reference's
own CPU build (oracle/_ref, through ckpt::restore after resizing its particle
array to the file's count) and steps it over the same steps.  Needs a GPU and
oracle/_ref; the reference takes about 7.5 s per step on 16 cores.

    python oracle/free_body_divergence.py --start 3540 --steps 40
"""
import argparse
import ctypes
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[0] = ROOT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--start", type=int, default=3540)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--restart", default="/tmp/free_body_restart.ckpt")
    args = ap.parse_args()
    import alebgk4paper_b200 as ab
    from oracle.oracle import RefCase, ref_library
    if ref_library() is None:
        sys.exit("oracle/_ref is not built (make -C oracle ref)")
    c = ab.Case("cavity3d-cube", 40, 10, -1.0, 2, fixed_body=False)
    s = ab.Solver(c, precision=64)
    st = c.bodies.copy()
    t0 = time.time()
    for _ in range(args.start):
        s.cudaStep(1)
        st = s.body_step(st)
        c.bodies = st
        s.refresh_geometry()
    print(f"device at step {args.start} after {time.time() - t0:.0f} s, N {c.N}", flush=True)
    s.checkpoint_save(args.restart, step=args.start, t=args.start * c.dt, bodies=st)
    g0, _ = s.cudaDownloadFull()
    dev, blow = {}, None
    for k in range(args.start + 1, args.start + args.steps + 1):
        s.cudaStep(1)
        st = s.body_step(st)
        c.bodies = st
        s.refresh_geometry()
        m = s.cudaDownloadMoments()
        dev[k] = (st[0, 3:6].copy(), float(np.nanmin(m[:, 0])), float(np.nanmax(m[:, 0])))
        if blow is None and (dev[k][2] > 10.0 or not np.isfinite(st).all()):
            blow = k
        if blow is not None and k >= blow + 3:
            break
    s.close()
    r = RefCase("cavity3d-cube", 40, 10, -1.0, 2, fixed_body=False)
    r.set_threads(os.cpu_count())
    r.L.ref_resize(r.h, int(g0.shape[0]))
    ok, step, _ = r.checkpoint_load(args.restart)
    cnt = (ctypes.c_int * 3)()
    r.L.ref_manage(r.h, cnt)          # neighbour lists of the restored cloud
    print(f"reference restored: {ok}, step {step}, distribution equal to the device's: "
          f"{bool(np.array_equal(r.g(), g0))}, management changes {list(cnt)}", flush=True)
    print("step | device: rho min, rho max, cube velocity | reference: the same", flush=True)
    for k in sorted(dev):
        r.step(1)
        m = r.macro()
        b = r.bodies()[0]
        v, lo, hi = dev[k]
        print(f"{k} | {lo:.6g} {hi:.6g} {np.round(v, 4)} | {m[:, 0].min():.6g} "
              f"{m[:, 0].max():.6g} {np.round(b[3:6], 4)}", flush=True)


if __name__ == "__main__":
    main()
