"""Batches of independent cavities on one B200, advanced by one CUDA graph
launch per step (``alebgk_batch_*`` of include/alebgk.h), and the seeded
batched-cavity2d workload: many lid-driven cavities of uneven resolution,
density and lid speed, each run to a steady residual.

The reference runs one cavity per process; there is no reference batch to
mirror, so this module only keeps the reference's per-cavity meaning (case
set-up TestCases/TestCases.cpp, the step of Solver/Solver.cpp:632-766).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from . import Case, LatticeCase, Solver, _check, _dp

__all__ = ["BatchSolver", "batched_cavity2d", "partition_lpt", "CAVITY2D_VMAX"]

# cavity2d's velocity grid extent (TestCases/TestCases.cpp:156)
CAVITY2D_VMAX = 1303.0


def batched_cavity2d(n: int = 96, seed: int = 0, Nx_choices=(24, 32, 40, 48),
                     Nv_choices=(16, 20, 24), lid=(0.5, 10.0), rho=(0.5, 11.0),
                     cfl: float = 1.25, mls_order: int = 2) -> list[dict]:
    """The seeded instance list of the batched cavity2d workload: Nx and Nv
    uniform over the choices, lid speed uniform, density log-uniform, the
    relaxation time scaled as 1/rho from the case's (TestCases.cpp:153, the
    hard-sphere scaling the reference applies between its cases), and dt at
    the given CFL of the fastest velocity node over the lattice spacing.

    CFL 1.25: the quadratic MLS transport is unstable at small CFL
    (TestCases.cpp:179-185 runs its 2-D body cases at CFL 1.3 for that
    reason).  At CFL 0.75 the cavities with Nv = 20 and 24 diverge after
    500-1500 steps, the reference's own CPU build included (Nx 24, Nv 24:
    density range 0.95-2.1 after 900 steps); at CFL 1.25 every (Nx, Nv) of
    the workload reaches the steady residual.  CFL 1.5 puts the fastest foot
    points on the stencil edge and diverges at once (Solver.cpp:175-179)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        Nx = int(rng.choice(Nx_choices))
        Nv = int(rng.choice(Nv_choices))
        u = float(rng.uniform(*lid))
        r = float(math.exp(rng.uniform(math.log(rho[0]), math.log(rho[1]))))
        dx = 1e-6 / (Nx - 1)
        out.append(dict(name="cavity2d", Nx=Nx, Nv=Nv, lid_speed=u, rho0=r,
                        tau=3.7142e-10 / r, dt=cfl * dx / CAVITY2D_VMAX,
                        mls_order=mls_order))
    return out


def partition_lpt(costs, nparts: int) -> list[list[int]]:
    """Longest-processing-time split of instances over nparts ranks: the
    costliest instance goes to the least loaded rank.  Deterministic."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * nparts
    parts: list[list[int]] = [[] for _ in range(nparts)]
    for i in order:
        r = min(range(nparts), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += costs[i]
    for p in parts:
        p.sort()
    return parts


class BatchSolver:
    """Independent cavities on one device, one graph launch per step.

    ``specs`` are keyword dictionaries for :class:`Case` (as
    :func:`batched_cavity2d` returns).  With ``autotune`` every cavity's
    launch shapes are tuned before the batch graph is captured.  With
    ``setup="device"`` each cavity's lattice, neighbour lists and rest state
    are built on the GPU (:class:`LatticeCase`) instead of on the host.

    ``launch="stages"`` (default) advances all cavities by one launch per
    stage of the step when they qualify (same precision and Chu layers,
    plain transport and particle kernels); ``launch="branches"`` puts every
    cavity's own step in the graph as a parallel branch.  Both compute each
    cavity exactly as it would step alone.

    ``residual="lid"`` measures each cavity's steady residual's momentum
    terms against its lid momentum rho U_lid (the spec's ``lid_speed``),
    ``residual="flow"`` against the flow's own momentum rho |u|, and
    ``residual="thermal"`` (the default) against the thermal momentum.
    """

    # launch forms: one launch per step stage in groups of cavities, every
    # cavity's own step as a graph branch, or the whole step in one
    # persistent cooperative launch
    _LAUNCH = {"stages": 0, "branches": 1, "persistent": 2}

    def __init__(self, specs, precision: int = 32, device: int = 0, autotune: bool = False,
                 tune_steps: int = 3, setup: str = "host", launch: str = "stages",
                 residual: str = "thermal"):
        if residual not in ("thermal", "lid", "flow"):
            raise ValueError("residual must be 'thermal', 'lid' or 'flow'")
        if setup not in ("host", "device"):
            raise ValueError("setup must be 'host' or 'device'")
        if launch not in self._LAUNCH:
            raise ValueError("launch must be 'stages', 'branches' or 'persistent'")
        self.lib = _abi.load()
        self.specs = list(specs)
        self.cases = []
        self.solvers = []
        for sp in self.specs:
            kw = dict(sp)
            name = kw.pop("name")
            c = LatticeCase(name, **kw) if setup == "device" else Case(name, **kw)
            self.cases.append(c)
            s = Solver(c, precision=precision, device=device)
            if residual == "lid":
                s.set_residual_speed(float(sp.get("lid_speed", 0.0)))
            elif residual == "flow":
                s.set_residual_speed(-1.0)
            self.solvers.append(s)
        self.tuned_ms = None
        if autotune:
            self.tuned_ms = [s.autotune(tune_steps) for s in self.solvers]
        n = len(self.solvers)
        arr = (ctypes.c_void_p * n)(*[s.ctx.value for s in self.solvers])
        h = ctypes.c_void_p()
        _check(self.lib.alebgk_batch_create(n, arr, ctypes.byref(h)), self.solvers[0].ctx)
        self.h = h
        self.steps = 0
        _check(self.lib.alebgk_batch_set_mode(self.h, self._LAUNCH[launch]),
               self.solvers[0].ctx)
        self.batch_tuned_ms = None
        if autotune:
            self.batch_tuned_ms = self.autotune(tune_steps)

    def autotune(self, steps: int = 3) -> float:
        """Times the batch's launch forms (stage launches in 1, 2, 4, 8
        groups; one persistent launch; per-cavity branches) and keeps the
        fastest.  The timed steps are real steps of the batch (every form
        computes the same states)."""
        ms = ctypes.c_float()
        _check(self.lib.alebgk_batch_autotune(self.h, int(steps), ctypes.byref(ms)),
               self.solvers[0].ctx)
        forms = 2 + sum(1 for g in (1, 2, 4, 8) if g <= len(self.solvers))
        self.steps += forms * (int(steps) + 2)
        return float(ms.value)

    @property
    def staged(self) -> int:
        """Stage groups of the step graph (0: per-cavity branches; known
        after the first step)."""
        mode, staged = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.alebgk_batch_get_mode(self.h, ctypes.byref(mode), ctypes.byref(staged)),
               self.solvers[0].ctx)
        return int(staged.value)

    def set_groups(self, groups: int):
        _check(self.lib.alebgk_batch_set_groups(self.h, int(groups)), self.solvers[0].ctx)

    def set_launch(self, launch: str):
        """Switches the launch form ('stages', 'branches', 'persistent')."""
        if launch not in self._LAUNCH:
            raise ValueError("launch must be 'stages', 'branches' or 'persistent'")
        _check(self.lib.alebgk_batch_set_mode(self.h, self._LAUNCH[launch]), self.solvers[0].ctx)

    @property
    def launch(self) -> str:
        mode, staged = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.alebgk_batch_get_mode(self.h, ctypes.byref(mode), ctypes.byref(staged)),
               self.solvers[0].ctx)
        return {v: k for k, v in self._LAUNCH.items()}[int(mode.value)]

    def set_spin_limit(self, polls: int):
        """Polls of the persistent launch's grid barrier before it gives up
        (sets bit 8 of the first cavity's error word and ends the step)."""
        _check(self.lib.alebgk_batch_set_spin_limit(self.h, int(polls)), self.solvers[0].ctx)

    @property
    def updates_per_step(self) -> int:
        return sum(c.N * c.gstride // (2 if c.dim == 2 else 1) for c in self.cases)

    def step(self, n: int = 1):
        _check(self.lib.alebgk_batch_step(self.h, int(n)), self.solvers[0].ctx)
        self.steps += n

    def sync(self):
        _check(self.lib.alebgk_batch_sync(self.h), self.solvers[0].ctx)

    def residuals(self) -> np.ndarray:
        out = np.zeros(len(self.solvers))
        _check(self.lib.alebgk_batch_residuals(self.h, _dp(out)), self.solvers[0].ctx)
        return out

    def interval_residuals(self) -> np.ndarray:
        """Per cavity the mean residual per step since the previous call
        (-1 on the first call)."""
        self.sync()
        return np.array([s.residual_interval() for s in self.solvers])

    def run_to_steady(self, tol: float = 1e-6, check_every: int = 50,
                      max_steps: int = 200000) -> np.ndarray:
        """Steps the batch until every cavity's mean residual per step over a
        check interval is below tol; returns per cavity the step count at
        the end of the first such interval (-1 if never).  Averaging over the
        interval keeps FP32 rounding noise of single steps (momentum noise
        of order 1e-7 of the thermal momentum, large against a slow flow's)
        out of the measure."""
        done = np.full(len(self.solvers), -1, np.int64)
        self.interval_residuals()
        while self.steps < max_steps and (done < 0).any():
            self.step(check_every)
            r = self.interval_residuals()
            newly = (r >= 0) & (r < tol) & (done < 0)
            done[newly] = self.steps
        return done

    def close(self):
        if getattr(self, "h", None):
            self.lib.alebgk_batch_destroy(self.h)
            self.h = None
        for s in getattr(self, "solvers", []):
            s.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
