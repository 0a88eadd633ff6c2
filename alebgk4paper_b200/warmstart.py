"""Learned warm start for 2-D lid-driven cavities.

A coordinate network predicts the 13-moment fields (rho, ux, uy, T,
sigma_xx, sigma_xy, sigma_yy, q_x, q_y) of a steady cavity from the particle
position and two case parameters, and the solver's distribution is seeded
from them by Grad's 13-moment expansion (``alebgk_seed_grad13``).  The
network is trained on steady states that the batched solver produces, by the
tensor-core kernels of ``csrc/warm.cu`` (``alebgk_net_*``).  The plain start
-- the Maxwellian at rest of Initialization/InitialConditions.cpp:18-80, with
which every case is built -- stays the fallback: a cavity is only seeded
when :func:`seed` is called.

The reference has no learned part; the moment definitions follow the
reference's 2-D Chu sums (MomentCalculations/Moments.cpp:66-97).

Targets are scaled per case so that they are of order one across the
workload's range of lid speeds and densities (Ma = U/c, c = sqrt(R Tw),
p0 = rho0 R Tw):

    (rho/rho0 - 1)/Ma, ux/U, uy/U, (T/Tw - 1)/Ma, sigma/(p0 Ma), q/(p0 c Ma)

and then standardised per channel with the training set's mean and spread,
which are stored with the weights.
"""
from __future__ import annotations

import ctypes
import json
import math
import time

import numpy as np

from . import _abi
from . import Case, Solver, _check

__all__ = ["WarmStartNet", "case_inputs", "case_targets", "denormalise", "seed",
           "moments13", "steady_dataset", "init_params", "RHO_RANGE", "LID_RANGE"]

N_PARAMS = 59920
N_OUT, N_USED = 16, 9
RHO_RANGE = (0.5, 11.0)
LID_RANGE = (0.5, 10.0)
CHANNELS = ("rho", "ux", "uy", "T", "sxx", "sxy", "syy", "qx", "qy")


def _lid_mach(case: Case) -> tuple[float, float]:
    U = case.params["lid_speed"]
    c = math.sqrt(case.params["R"] * case.params["Tw"])
    return U / c, c


def case_inputs(case: Case) -> np.ndarray:
    """Network input rows (x/L, y/L, a, b) of every particle of a 2-D case:
    a the log density and b the lid Mach number, both mapped to [-1, 1]
    over the workload's ranges."""
    p = case.params
    x = (case.xyz[:, 0] - p["xleft"]) / (p["xright"] - p["xleft"])
    y = (case.xyz[:, 1] - p["ybottom"]) / (p["ytop"] - p["ybottom"])
    lo, hi = math.log(RHO_RANGE[0]), math.log(RHO_RANGE[1])
    a = (2 * math.log(p["rho0"]) - lo - hi) / (hi - lo)
    c = math.sqrt(p["R"] * p["Tw"])
    mlo, mhi = LID_RANGE[0] / c, LID_RANGE[1] / c
    b = (2 * _lid_mach(case)[0] - mlo - mhi) / (mhi - mlo)
    out = np.empty((case.N, 4), np.float32)
    out[:, 0], out[:, 1], out[:, 2], out[:, 3] = x, y, a, b
    return out


def _case_scales(case: Case):
    """Per-channel (offset, unit) of the scaled targets: m = offset + unit * t."""
    p = case.params
    Ma, c = _lid_mach(case)
    U, rho0, Tw = p["lid_speed"], p["rho0"], p["Tw"]
    p0 = rho0 * p["R"] * Tw
    off = np.array([rho0, 0, 0, Tw, 0, 0, 0, 0, 0], np.float64)
    unit = np.array([rho0 * Ma, U, U, Tw * Ma, p0 * Ma, p0 * Ma, p0 * Ma,
                     p0 * c * Ma, p0 * c * Ma], np.float64)
    return off, unit


def case_targets(case: Case, mom: np.ndarray) -> np.ndarray:
    """Scaled targets (N, 9) of 13-moment rows (N, 9) of a case."""
    off, unit = _case_scales(case)
    return ((mom - off) / unit).astype(np.float32)


def denormalise(case: Case, mu: np.ndarray, sd: np.ndarray):
    """(scale, shift) with moments = shift + scale * network output."""
    off, unit = _case_scales(case)
    return unit * sd, off + unit * mu


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases (rows 9..15 of the output layer 0)."""
    rng = np.random.default_rng(seed)
    shapes = [(64, 128), (128, 128), (128, 128), (128, 128), (128, 16)]
    out = []
    for l, (i, o) in enumerate(shapes):
        a = math.sqrt(6.0 / (i + o))
        w = rng.uniform(-a, a, size=(o, i)).astype(np.float32)
        if l == 4:
            w[N_USED:] = 0
        out.append(w.ravel())
    out.append(np.zeros(4 * 128 + 16, np.float32))
    p = np.concatenate(out)
    assert p.size == N_PARAMS
    return p


def _pad16(T):
    """Target rows widened to the network's 16 outputs (numpy input)."""
    if isinstance(T, np.ndarray) and T.shape[1] < N_OUT:
        out = np.zeros((T.shape[0], N_OUT), np.float32)
        out[:, :T.shape[1]] = T
        return out
    return T


class WarmStartNet:
    """The coordinate network on one device (``alebgk_net``)."""

    def __init__(self, params: np.ndarray | None = None, mu=None, sd=None, device: int = 0,
                 seed: int = 0):
        import torch
        self.torch = torch
        self.lib = _abi.load()
        assert self.lib.alebgk_net_nparams() == N_PARAMS
        self.device = device
        self.meta = {}
        h = ctypes.c_void_p()
        rc = self.lib.alebgk_net_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"alebgk_net_create failed ({rc})")
        self.h = h
        self.mu = np.zeros(N_USED) if mu is None else np.asarray(mu, np.float64)
        self.sd = np.ones(N_USED) if sd is None else np.asarray(sd, np.float64)
        self.set_params(init_params(seed) if params is None else params)

    # -- parameters ----------------------------------------------------------
    def _ok(self, rc):
        if rc != 0:
            msg = self.lib.alebgk_net_last_error(self.h)
            raise RuntimeError(f"alebgk error {rc}: {msg.decode() if msg else ''}")

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        assert p.shape == (N_PARAMS,)
        self._ok(self.lib.alebgk_net_set_params(self.h, p.ctypes.data_as(_abi.c_float_p)))

    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        self._ok(self.lib.alebgk_net_get_params(self.h, p.ctypes.data_as(_abi.c_float_p)))
        return p

    def save(self, path: str, meta: dict | None = None):
        np.savez(path, params=self.params(), mu=self.mu, sd=self.sd,
                 meta=json.dumps(meta or self.meta))

    @classmethod
    def load(cls, path: str, device: int = 0) -> "WarmStartNet":
        d = np.load(path)
        net = cls(d["params"], d["mu"], d["sd"], device=device)
        net.meta = json.loads(str(d["meta"]))
        return net

    # -- device calls --------------------------------------------------------
    def _dev(self, a, dtype):
        t = self.torch
        if isinstance(a, t.Tensor):
            return a.to(device=f"cuda:{self.device}", dtype=dtype).contiguous()
        return t.as_tensor(np.ascontiguousarray(a), dtype=dtype,
                           device=f"cuda:{self.device}").contiguous()

    def forward(self, pts, idx=None):
        """Network outputs (n, 16) FP32 on the device for input rows (n, 4)."""
        t = self.torch
        x = self._dev(pts, t.float32)
        n = x.shape[0] if idx is None else len(idx)
        ix = None if idx is None else self._dev(idx, t.int32)
        out = t.empty((n, N_OUT), dtype=t.float32, device=x.device)
        self._ok(self.lib.alebgk_net_forward(self.h, x.data_ptr(),
                                             None if ix is None else ix.data_ptr(), n,
                                             out.data_ptr()))
        return out

    def grad(self, pts, tgt, idx=None, chan_w=None):
        """(loss, gradient) of the weighted squared error over the batch."""
        t = self.torch
        x, y = self._dev(pts, t.float32), self._dev(_pad16(tgt), t.float32)
        n = x.shape[0] if idx is None else len(idx)
        ix = None if idx is None else self._dev(idx, t.int32)
        w = np.ones(N_USED, np.float32) if chan_w is None else np.asarray(chan_w, np.float32)
        g = np.zeros(N_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._ok(self.lib.alebgk_net_grad(self.h, x.data_ptr(), y.data_ptr(),
                                          None if ix is None else ix.data_ptr(), n,
                                          w.ctypes.data_as(_abi.c_float_p),
                                          g.ctypes.data_as(_abi.c_float_p), ctypes.byref(loss)))
        return loss.value, g

    def fit(self, X, T, steps: int = 4000, batch: int = 16384, lr: float = 2e-3,
            lr_final: float = 5e-5, seed: int = 0, log_every: int = 500, chan_w=None):
        """Adam on mini-batches drawn without replacement per epoch; cosine
        learning-rate decay from lr to lr_final.  Returns the logged losses
        (weighted squared error per row)."""
        t = self.torch
        x, y = self._dev(X, t.float32), self._dev(_pad16(T), t.float32)
        n = x.shape[0]
        batch = min(batch, n)
        rng = np.random.default_rng(seed)
        w = np.ones(N_USED, np.float32) if chan_w is None else np.asarray(chan_w, np.float32)
        wp = w.ctypes.data_as(_abi.c_float_p)
        perm, pos, log = None, n, []
        for s in range(steps):
            if pos + batch > n:
                perm = self._dev(rng.permutation(n).astype(np.int32), t.int32)
                pos = 0
            ix = perm[pos:pos + batch]
            pos += batch
            cur = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * s / max(1, steps)))
            want = bool(log_every) and (s % log_every == 0 or s == steps - 1)
            loss = ctypes.c_float()
            self._ok(self.lib.alebgk_net_train_step(
                self.h, x.data_ptr(), y.data_ptr(), ix.data_ptr(), int(ix.shape[0]), wp,
                float(cur), 0.9, 0.999, 1e-8, ctypes.byref(loss) if want else None))
            if want:
                log.append((s, loss.value / ix.shape[0]))
        self._ok(self.lib.alebgk_net_sync(self.h))
        return log

    def close(self):
        if getattr(self, "h", None):
            self.lib.alebgk_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def moments13(solver: Solver) -> np.ndarray:
    """13-moment rows (N, 9) FP64 of a 2-D solver's current state."""
    import torch
    out = torch.empty((solver.N, 9), dtype=torch.float64, device=f"cuda:{solver.cfg.device}")
    _check(solver.lib.alebgk_moments13(solver.ctx, out.data_ptr()), solver.ctx)
    return out.cpu().numpy()


def seed(solver: Solver, net: WarmStartNet, case: Case | None = None):
    """Seeds a 2-D solver's state from the network's prediction for its case."""
    case = case if case is not None else solver.case
    out = net.forward(case_inputs(case))
    scale, shift = denormalise(case, net.mu, net.sd)
    scale = np.ascontiguousarray(scale, np.float64)
    shift = np.ascontiguousarray(shift, np.float64)
    _check(solver.lib.alebgk_seed_grad13(solver.ctx, out.data_ptr(), N_OUT,
                                         scale.ctypes.data_as(_abi.c_double_p),
                                         shift.ctypes.data_as(_abi.c_double_p)), solver.ctx)


def steady_dataset(specs, tol: float = 1e-6, check_every: int = 25, max_steps: int = 20000,
                   chunk: int = 96, precision: int = 32, device: int = 0, settle: int = 0,
                   verbose=False):
    """Runs batches of cavities to the steady residual, then `settle` more
    steps (the residual tolerance leaves the slow modes a few percent from
    their limit), and returns per case a dict: inputs (N, 4), mom (N, 9)
    13-moment rows, targets (N, 9) scaled, steps to steady (-1 if never)."""
    from .batch import BatchSolver
    out = []
    for a in range(0, len(specs), chunk):
        part = specs[a:a + chunk]
        t0 = time.perf_counter()
        b = BatchSolver(part, precision=precision, device=device)
        done = b.run_to_steady(tol=tol, check_every=check_every, max_steps=max_steps)
        if settle:
            b.step(settle)
            b.sync()
        for s, c, d in zip(b.solvers, b.cases, done):
            m = moments13(s)
            out.append(dict(inputs=case_inputs(c), mom=m, targets=case_targets(c, m),
                            steps=int(d)))
        steps = b.steps
        b.close()
        if verbose:
            print(f"steady batch {a // chunk}: {len(part)} cases, {steps} steps, "
                  f"{time.perf_counter() - t0:.1f} s, unsteady {(done < 0).sum()}", flush=True)
    return out
