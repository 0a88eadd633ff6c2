"""Slab mode: one large cavity split into slabs along its outermost lattice
axis (z in 3-D, y in 2-D), one context per slab (``alebgk_slab_*``).

The plan restates the reference's decomposed mode
(Solver/MpiExchange.cpp:199-318): rows [r0, r1) = [s R / n, (s+1) R / n)
per slab, ghost rows ceil(radius / spacing) + 1 on each inner side, every
slab at least two halos tall.  A slab keeps the global particle order, so its
owned particles are one contiguous range and its neighbour lists are the
global lists renumbered (owned particles see all their neighbours; ghost
rows keep only those inside the slab, and are refreshed from their owners
after every step instead of being trusted).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from . import Case, Solver, _check, _dp

__all__ = ["plan_slabs", "SlabGroup", "RankSlab", "rank_halo_plan"]


def _rows(case):
    """(rows along the slab axis, particles per row, row spacing)."""
    p = case.params
    if case.dim == 3:
        nz = int(round((p["zback"] - p["zfront"]) / p["dz"])) + 1
        return nz, case.N // nz, abs(p["dz"])
    ny = int(round((p["ytop"] - p["ybottom"]) / p["dy"])) + 1
    return ny, case.N // ny, abs(p["dy"])


def plan_slabs(case, nslabs: int) -> dict:
    """The slab layout of a lattice case: per slab the kept global rows
    [k0, k1), the owned rows [r0, r1), the owned local particle range and
    the ghost copies (dst slab, dst start, src slab, src start, count)."""
    if case.nbodies:
        raise ValueError("slab mode takes box cavities without bodies")
    R, stride, spacing = _rows(case)
    if R * stride != case.N:
        raise ValueError("the cloud is not a complete lattice")
    halo = int(math.ceil(case.params["radius"] / spacing)) + 1
    slabs = []
    for s in range(nslabs):
        r0, r1 = s * R // nslabs, (s + 1) * R // nslabs
        if r1 - r0 < 2 * halo:
            raise ValueError(f"slab {s} has {r1 - r0} rows; slab mode needs at least "
                             f"{2 * halo} (two halos of {halo})")
        k0 = max(0, r0 - halo) if s > 0 else 0
        k1 = min(R, r1 + halo) if s < nslabs - 1 else R
        slabs.append(dict(r0=r0, r1=r1, k0=k0, k1=k1,
                          own=((r0 - k0) * stride, (r1 - k0) * stride)))
    copies = []
    for s, sl in enumerate(slabs):
        if s > 0:                 # ghosts below <- slab s-1's top owned rows
            nb = slabs[s - 1]
            copies.append((s, 0, s - 1, (sl["k0"] - nb["k0"]) * stride,
                           (sl["r0"] - sl["k0"]) * stride))
        if s < nslabs - 1:        # ghosts above <- slab s+1's bottom owned rows
            nb = slabs[s + 1]
            copies.append((s, (sl["r1"] - sl["k0"]) * stride, s + 1,
                           (sl["r1"] - nb["k0"]) * stride, (sl["k1"] - sl["r1"]) * stride))
    return dict(rows=R, stride=stride, halo=halo, slabs=slabs, copies=copies)


class _SlabCase:
    """The particles of one slab as a case a :class:`Solver` can upload."""

    config = Case.config
    cloud = Case.cloud

    def __init__(self, case, k0: int, k1: int, stride: int):
        a, b = k0 * stride, k1 * stride
        self.name = case.name
        self.dim, self.Nv, self.gstride = case.dim, case.Nv, case.gstride
        self.mls_order, self.params, self.dt = case.mls_order, case.params, case.dt
        self.nbodies = 0
        self.N = b - a
        self.xyz = case.xyz[a:b].copy()
        self.meshv = case.meshv[a:b].copy()
        self.wall = case.wall[a:b].copy()
        self.boundary = case.boundary[a:b].copy()
        self.body_id = case.body_id[a:b].copy()
        self.g = case.g[a:b].copy()
        self.macro = case.macro[a:b].copy()
        nbr = np.full((self.N, _abi.MAX_NEIGH), -1, np.int32)
        nnb = np.zeros(self.N, np.int32)
        for i in range(self.N):
            row = case.nbr[a + i, :case.nnb[a + i]]
            keep = row[(row >= a) & (row < b)] - a
            nbr[i, :len(keep)] = keep
            nnb[i] = len(keep)
        self.nbr, self.nnb = nbr, nnb


class SlabGroup:
    """A lattice case stepped as ``nslabs`` slabs (one context each)."""

    def __init__(self, case, nslabs: int, precision: int = 32, devices=None):
        self.lib = _abi.load()
        self.case = case
        self.plan = plan_slabs(case, nslabs)
        devices = devices or [0] * nslabs
        st = self.plan["stride"]
        self.subcases, self.solvers = [], []
        for s, sl in enumerate(self.plan["slabs"]):
            sc = _SlabCase(case, sl["k0"], sl["k1"], st)
            self.subcases.append(sc)
            self.solvers.append(Solver(sc, precision=precision, device=devices[s]))
        n = nslabs
        ctxs = (ctypes.c_void_p * n)(*[s.ctx.value for s in self.solvers])
        lo = np.array([sl["own"][0] for sl in self.plan["slabs"]], np.int32)
        hi = np.array([sl["own"][1] for sl in self.plan["slabs"]], np.int32)
        cp = np.array(self.plan["copies"], np.int32).reshape(-1, 5)
        h = ctypes.c_void_p()
        _check(self.lib.alebgk_slab_create(n, ctxs, lo.ctypes.data_as(_abi.c_int_p),
                                           hi.ctypes.data_as(_abi.c_int_p), len(cp),
                                           cp.ctypes.data_as(_abi.c_int_p), ctypes.byref(h)),
               self.solvers[0].ctx)
        self.h = h
        self.steps = 0

    def step(self, n: int = 1):
        _check(self.lib.alebgk_slab_step(self.h, int(n)), self.solvers[0].ctx)
        self.steps += n

    def sync(self):
        _check(self.lib.alebgk_slab_sync(self.h), self.solvers[0].ctx)

    def download_full(self):
        """The whole cavity's (g, macro) assembled from the slabs' owned rows,
        in the global particle order."""
        self.sync()
        st = self.plan["stride"]
        g = np.zeros((self.case.N, self.case.gstride))
        m = np.zeros((self.case.N, 7))
        for s, sl in zip(self.solvers, self.plan["slabs"]):
            gs, ms = s.cudaDownloadFull()
            lo, hi = sl["own"]
            g[sl["r0"] * st:sl["r1"] * st] = gs[lo:hi]
            m[sl["r0"] * st:sl["r1"] * st] = ms[lo:hi]
        return g, m

    def total_mass(self) -> float:
        return self.solvers[0].cudaTotalMass()

    def close(self):
        if getattr(self, "h", None):
            self.lib.alebgk_slab_destroy(self.h)
            self.h = None
        for s in getattr(self, "solvers", []):
            s.cudaFreeCloud()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rank_halo_plan(plan: dict, rank: int):
    """This rank's part of the ghost copies: (sends, receives), each a list
    of (peer rank, local start, count) -- sends read the rank's own rows,
    receives write its ghost rows (MpiExchange.cpp:405-466)."""
    sends, recvs = [], []
    for dst, dst_start, src, src_start, count in plan["copies"]:
        if src == rank:
            sends.append((dst, src_start, count))
        if dst == rank:
            recvs.append((src, dst_start, count))
    return sends, recvs


class RankSlab:
    """One slab of a lattice cavity per process of a ``torch.distributed``
    group: the reference's MPI decomposed mode (Solver/MpiExchange.cpp:
    199-466).  Rank r steps slab r of ``plan_slabs(case, world)``.  Between
    the four segments of a step the slabs' combine words (owned-range partial
    sums and the moodCheck flag) are all-gathered in rank order
    (MomentCalculations/Conservation.cpp:33-36,76-84); after the last
    segment the ghost rows are exchanged with the neighbouring ranks.  The
    combine is the single-process slab group's, so the run gives that
    group's state.  The exchanges go through host buffers, as CPU tensors for
    ``gloo`` and as device tensors for ``nccl``.

    ``lib`` and ``solver_factory`` default to the compiled library and
    :class:`Solver`; tests replace them."""

    def __init__(self, case, precision: int = 32, device: int = 0, group=None, lib=None,
                 solver_factory=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.plan = plan_slabs(case, self.world)
        st = self.plan["stride"]
        sl = self.plan["slabs"][self.rank]
        self.sub = _SlabCase(case, sl["k0"], sl["k1"], st)
        self.lib = lib or _abi.load()
        make = solver_factory or (lambda c: Solver(c, precision=precision, device=device))
        self.solver = make(self.sub)
        self.ctx = self.solver.ctx
        self.own = sl["own"]
        self.sends, self.recvs = rank_halo_plan(self.plan, self.rank)
        ldf, es = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.alebgk_device_state(self.ctx, None, ctypes.byref(ldf), ctypes.byref(es)),
               self.ctx)
        self.row_bytes = ldf.value * es.value
        self.device = device
        words = np.zeros(4)
        _check(self.lib.alebgk_rank_slab_init(self.ctx, self.world, int(self.own[0]),
                                              int(self.own[1]), _dp(words)), self.ctx)
        self._combine(4, words)
        self.steps = 0

    def _nccl(self) -> bool:
        return self.dist.get_backend(self.group) == "nccl"

    def _tensor(self, a):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.cuda(self.device) if self._nccl() else t

    def _combine(self, phase: int, words: np.ndarray):
        import torch
        mine = self._tensor(words.astype(np.float64))
        out = [torch.zeros_like(mine) for _ in range(self.world)]
        self.dist.all_gather(out, mine, group=self.group)
        allw = np.concatenate([o.cpu().numpy() for o in out]).astype(np.float64)
        _check(self.lib.alebgk_rank_slab_combine(self.ctx, int(phase), self.world, _dp(allw)),
               self.ctx)

    def _rows(self, start: int, count: int, f=None, m=None, put: bool = False):
        if f is None:
            f = np.zeros(count * self.row_bytes, np.uint8)
            m = np.zeros(count * 6)
        _check(self.lib.alebgk_rank_slab_rows(self.ctx, int(start), int(count),
                                              f.ctypes.data_as(ctypes.c_void_p), _dp(m),
                                              1 if put else 0), self.ctx)
        return f, m

    def _halo(self):
        """Ghost rows of the state being written, from their owners.

        Every receive and send of the exchange is posted in one
        batch_isend_irecv call.  Under NCCL that call groups the point-to-point
        operations, so two ranks that each receive from and send to the other
        cannot deadlock on the order in which their operations were queued on
        the communicator's stream; under gloo it posts them one by one."""
        import torch
        ops, inbox, keep = [], [], []
        P2POp = self.dist.P2POp
        for peer, start, count in self.recvs:
            f = self._tensor(np.zeros(count * self.row_bytes, np.uint8))
            m = self._tensor(np.zeros(count * 6))
            ops += [P2POp(self.dist.irecv, f, peer, self.group),
                    P2POp(self.dist.irecv, m, peer, self.group)]
            inbox.append((start, count, f, m))
        for peer, start, count in self.sends:
            f, m = self._rows(start, count)
            tf, tm = self._tensor(f), self._tensor(m)
            keep.append((tf, tm))
            ops += [P2POp(self.dist.isend, tf, peer, self.group),
                    P2POp(self.dist.isend, tm, peer, self.group)]
        for r in (self.dist.batch_isend_irecv(ops) if ops else []):
            r.wait()
        for start, count, f, m in inbox:
            fh = np.ascontiguousarray(f.cpu().numpy())
            mh = np.ascontiguousarray(m.cpu().numpy()).astype(np.float64)
            self._rows(start, count, fh, mh, put=True)
        del keep, torch

    def step(self, n: int = 1):
        for _ in range(int(n)):
            for seg in range(4):
                words = np.zeros(4)
                _check(self.lib.alebgk_rank_slab_segment(self.ctx, seg, _dp(words)), self.ctx)
                self._combine(seg, words)
            self._halo()
            _check(self.lib.alebgk_rank_slab_finish(self.ctx), self.ctx)
            self.steps += 1

    def owned(self):
        """This rank's owned rows of (g, macro) and their global row range."""
        g, m = self.solver.cudaDownloadFull()
        lo, hi = self.own
        sl = self.plan["slabs"][self.rank]
        st = self.plan["stride"]
        return g[lo:hi], m[lo:hi], (sl["r0"] * st, sl["r1"] * st)

    def close(self):
        if getattr(self, "solver", None) is not None:
            self.solver.close()
            self.solver = None
