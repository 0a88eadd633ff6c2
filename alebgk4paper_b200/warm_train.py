"""Training and evaluation of the learned warm start (``python -m
alebgk4paper_b200.warm_train``).

1. Steady states: seeded batched-cavity2d instances (Nx in {24, 32, 40, 48},
   Nv in {16, 20, 24}, lid speed and density drawn as in
   :func:`alebgk4paper_b200.batch.batched_cavity2d`) are run by the batched
   solver from the Maxwellian at rest to the steady residual, and their
   13-moment fields are read back (``alebgk_moments13``).
2. Training: the coordinate network is fitted to the scaled fields by the
   tensor-core kernels (``alebgk_net_train_step``), Adam with cosine decay.
3. Evaluation on held-out seeded cases at Nx = 48, Nv = 20: every case runs
   to the steady residual once from the plain start and once seeded by the
   network; steps, wall time and the difference of the two steady states are
   reported.

The inputs are the solver's own steady states; there is no external data.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .batch import BatchSolver, batched_cavity2d
from . import warmstart as ws

DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                             "warmstart_cavity2d.npz")
TRAIN_SEED, HELDOUT_SEED = 1000, 2000


def training_specs(n: int = 2000, seed: int = TRAIN_SEED):
    return batched_cavity2d(n, seed=seed)


def heldout_specs(n: int = 32, seed: int = HELDOUT_SEED, Nx: int = 48, Nv: int = 20):
    return batched_cavity2d(n, seed=seed, Nx_choices=(Nx,), Nv_choices=(Nv,))


def build_dataset(specs, chunk: int = 96, check_every: int = 25, settle: int = 3000,
                  verbose: bool = True):
    """Concatenated inputs (P, 4), scaled targets (P, 9) and the per-case
    records of the steady runs."""
    recs = ws.steady_dataset(specs, check_every=check_every, chunk=chunk, settle=settle,
                             verbose=verbose)
    X = np.concatenate([r["inputs"] for r in recs])
    T = np.concatenate([r["targets"] for r in recs])
    return X, T, recs


def train(X, T, steps: int = 20000, batch: int = 16384, lr: float = 2e-3,
          lr_final: float = 2e-5, seed: int = 0, verbose: bool = True):
    """A network fitted to (X, T), with the channel statistics of T."""
    mu = T.mean(0).astype(np.float64)
    sd = T.std(0).astype(np.float64)
    sd[sd < 1e-12] = 1.0
    Tn = ((T - mu) / sd).astype(np.float32)
    net = ws.WarmStartNet(mu=mu, sd=sd, seed=seed)
    t0 = time.perf_counter()
    log = net.fit(X, Tn, steps=steps, batch=batch, lr=lr, lr_final=lr_final, seed=seed,
                  log_every=max(1, steps // 20))
    net.meta = dict(train_seconds=time.perf_counter() - t0, steps=steps, batch=batch,
                    points=int(len(X)), loss_log=[(int(s), float(l)) for s, l in log])
    if verbose:
        for s, l in log:
            print(f"  step {s:6d}  loss/row {l:.4e}", flush=True)
    return net


def _run(specs, net=None, tol: float = 5e-7, check_every: int = 200, max_steps: int = 60000,
         residual: str = "lid"):
    """Runs the cases to steady, cold or seeded; returns (steps per case,
    seconds until all are steady incl. seeding, 13-moment rows per case).
    Steady: the mean change per step over a check interval, momentum against
    the lid momentum (residual="lid"), below tol."""
    b = BatchSolver(specs, residual=residual)
    b.sync()
    t0 = time.perf_counter()
    if net is not None:
        for s, c in zip(b.solvers, b.cases):
            ws.seed(s, net, c)
    done = b.run_to_steady(tol=tol, check_every=check_every, max_steps=max_steps)
    b.sync()
    sec = time.perf_counter() - t0
    moms = [ws.moments13(s) for s in b.solvers]
    cases = b.cases
    pred = None
    if net is not None:
        pred = []
        for c in cases:
            out = net.forward(ws.case_inputs(c)).cpu().numpy()[:, :9].astype(np.float64)
            scale, shift = ws.denormalise(c, net.mu, net.sd)
            pred.append(shift + scale * out)
    b.close()
    return done, sec, moms, pred


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _reference(specs, steps: int):
    """13-moment rows after a fixed, long cold run: the converged fields the
    steady states at the residual tolerance are measured against."""
    b = BatchSolver(specs)
    b.step(steps)
    b.sync()
    moms = [ws.moments13(s) for s in b.solvers]
    b.close()
    return moms


def evaluate(net, specs, tol: float = 5e-7, check_every: int = 200, max_steps: int = 60000,
             reference_steps: int = 8000, residual: str = "lid"):
    """Cold start against warm start on the same cases; both steady states
    are also compared with the fields after a long cold run."""
    cold, t_cold, m_cold, _ = _run(specs, None, tol, check_every, max_steps, residual)
    warm, t_warm, m_warm, pred = _run(specs, net, tol, check_every, max_steps, residual)
    m_ref = _reference(specs, reference_steps) if reference_steps else None
    names = ("rho", "ux", "uy", "T")
    field = {k: [] for k in names}
    dev = {k: [] for k in ("rho", "T")}
    for mc, mw, mp, sp in zip(m_cold, m_warm, pred, specs):
        for j, k in enumerate(names):
            field[k].append(_rel(mw[:, j], mc[:, j]))
        ref = np.array([sp["rho0"], 270.0])
        for j, k in ((0, "rho"), (3, "T")):
            base = ref[0] if k == "rho" else ref[1]
            dev[k].append(float(np.linalg.norm(mw[:, j] - mc[:, j]) /
                                max(np.linalg.norm(mc[:, j] - base), 1e-300)))
    chan = ws.CHANNELS
    pred_all = {k: float(np.median([_rel(mp[:, j], mc[:, j]) for mp, mc in zip(pred, m_cold)]))
                for j, k in enumerate(chan)}
    vs_ref = None
    if m_ref is not None:
        vs_ref = {}
        for tag, ms in (("cold", m_cold), ("warm", m_warm)):
            vs_ref[tag] = {k: max(_rel(m[:, j], mr[:, j]) for m, mr in zip(ms, m_ref))
                           for j, k in enumerate(names)}
        vs_ref["reference_steps"] = reference_steps
    ok = (cold > 0) & (warm > 0)
    return {
        "cases": len(specs), "tol": tol, "check_every": check_every, "residual": residual,
        "cold_steps": cold.tolist(), "warm_steps": warm.tolist(),
        "cold_steps_mean": float(cold[ok].mean()) if ok.any() else None,
        "warm_steps_mean": float(warm[ok].mean()) if ok.any() else None,
        "steps_ratio": float(cold[ok].sum() / max(1, warm[ok].sum())) if ok.any() else None,
        "cold_seconds": t_cold, "warm_seconds": t_warm,
        "wall_ratio": t_cold / t_warm if t_warm > 0 else None,
        "all_steady": bool(ok.all()),
        "field_rel_err_max": {k: max(v) for k, v in field.items()},
        "field_rel_err_median": {k: float(np.median(v)) for k, v in field.items()},
        "deviation_rel_err_max": {k: max(v) for k, v in dev.items()},
        "prediction_rel_err_median": pred_all,
        "vs_converged_max": vs_ref,
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--heldout", type=int, default=32)
    ap.add_argument("--settle", type=int, default=3000)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-only", action="store_true")
    args = ap.parse_args(argv)
    report = {}
    if args.eval_only:
        net = ws.WarmStartNet.load(args.out)
    else:
        t0 = time.perf_counter()
        X, T, recs = build_dataset(training_specs(args.cases), settle=args.settle)
        steady = np.array([r["steps"] for r in recs])
        report["data"] = dict(cases=len(recs), points=int(len(X)),
                              seconds=time.perf_counter() - t0,
                              unsteady=int((steady < 0).sum()),
                              steps_mean=float(steady[steady > 0].mean()))
        print(json.dumps(report["data"]), flush=True)
        net = train(X, T, steps=args.steps, batch=args.batch)
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        net.meta.update(report["data"])
        net.save(args.out)
        report["train"] = {k: v for k, v in net.meta.items() if k != "loss_log"}
        report["train"]["final_loss"] = net.meta["loss_log"][-1][1]
    report["eval"] = evaluate(net, heldout_specs(args.heldout))
    print(json.dumps(report["eval"]), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
