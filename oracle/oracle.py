"""TEST INFRASTRUCTURE ONLY: Python access to the two CPU checkers.

* :class:`Oracle` -- the plain-C FP64 restatement in ``alebgk_oracle.c``
  (``oracle/_build/liboracle.so``), run on a cloud given as numpy arrays.
* :class:`RefCase` -- the reference's own CPU sources compiled unmodified into
  ``oracle/_ref/libalebgk_ref_<isa>.so`` (see ``oracle/Makefile``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
legs of ``bench.py`` import this module.  The product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
MAX_NEIGH = 128

_vp = ctypes.c_void_p


def _p(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def build_oracle() -> str:
    """Compiles liboracle.so with gcc if missing (works without the reference)."""
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return ORACLE_LIB


class _OraCloud(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("N", ctypes.c_int), ("Nv", ctypes.c_int), ("gs", ctypes.c_int),
        ("mls_order", ctypes.c_int), ("limiter", ctypes.c_int), ("tau_variable", ctypes.c_int),
        ("dt", ctypes.c_double), ("tau", ctypes.c_double), ("R", ctypes.c_double),
        ("dHS", ctypes.c_double), ("vmin", ctypes.c_double), ("dv", ctypes.c_double),
        ("h", ctypes.c_double),
        ("periodic", ctypes.c_int * 3), ("L", ctypes.c_double * 3),
        ("xyz", _vp), ("meshv", _vp), ("wall", _vp),
        ("boundary", _vp), ("body_id", _vp), ("nnb", _vp), ("nbr", _vp),
        ("g", _vp), ("gt", _vp), ("macro", _vp), ("flag", _vp),
    ]


class _OraStats(ctypes.Structure):
    _fields_ = [("transport_flags", ctypes.c_int), ("mood_fail", ctypes.c_int),
                ("positivity_fixes", ctypes.c_int), ("mass_old", ctypes.c_double),
                ("mass_new", ctypes.c_double), ("mass_end", ctypes.c_double)]


class Oracle:
    """FP64 CPU restatement stepping its own copy of a cloud."""

    def __init__(self, *, dim, Nv, dt, tau, R, dHS, vmin, dv, h, xyz, meshv, wall,
                 boundary, body_id, nnb, nbr, g, macro, mls_order=2, limiter=2,
                 tau_variable=0):
        self.lib = ctypes.CDLL(build_oracle())
        N = len(boundary)
        self.N, self.dim, self.Nv = N, dim, Nv
        self.gs = Nv ** 3 if dim == 3 else 2 * Nv * Nv
        self.xyz = np.ascontiguousarray(xyz, np.float64).copy()
        self.meshv = np.ascontiguousarray(meshv, np.float64).copy()
        self.wall = np.ascontiguousarray(wall, np.float64).copy()
        self.boundary = np.ascontiguousarray(boundary, np.int32).copy()
        self.body_id = np.ascontiguousarray(body_id, np.int32).copy()
        self.nnb = np.ascontiguousarray(nnb, np.int32).copy()
        self.nbr = np.ascontiguousarray(nbr, np.int32).reshape(N, MAX_NEIGH).copy()
        self.g = np.ascontiguousarray(g, np.float64).reshape(N, self.gs).copy()
        self.gt = np.zeros_like(self.g)
        self.macro = np.ascontiguousarray(macro, np.float64).reshape(N, 7).copy()
        self.flag = np.zeros(N, np.int32)
        c = _OraCloud()
        c.dim, c.N, c.Nv, c.gs = dim, N, Nv, self.gs
        c.mls_order, c.limiter, c.tau_variable = mls_order, limiter, tau_variable
        c.dt, c.tau, c.R, c.dHS, c.vmin, c.dv, c.h = dt, tau, R, dHS, vmin, dv, h
        for a, arr in (("xyz", self.xyz), ("meshv", self.meshv), ("wall", self.wall),
                       ("boundary", self.boundary), ("body_id", self.body_id),
                       ("nnb", self.nnb), ("nbr", self.nbr), ("g", self.g),
                       ("gt", self.gt), ("macro", self.macro), ("flag", self.flag)):
            setattr(c, a, _p(arr))
        self.c = c
        self.stats = {}

    @classmethod
    def from_case(cls, case, **kw):
        p = case.params
        return cls(dim=case.dim, Nv=case.Nv, dt=kw.pop("dt", case.dt), tau=p["tau"],
                   R=p["R"], dHS=p["dHS"], vmin=p["vmin"], dv=p["dv"], h=p["radius"],
                   xyz=case.xyz, meshv=case.meshv, wall=case.wall, boundary=case.boundary,
                   body_id=case.body_id, nnb=case.nnb, nbr=case.nbr, g=case.g,
                   macro=case.macro, mls_order=kw.pop("mls_order", case.mls_order), **kw)

    def step(self, n=1):
        st = _OraStats()
        self.lib.ora_step(ctypes.byref(self.c), int(n), ctypes.byref(st))
        self.stats = {k: getattr(st, k) for k, _ in _OraStats._fields_}
        return self.stats

    def transport(self):
        """Transport + MOOD screen + linear redo into gt (no commit)."""
        nfix = ctypes.c_int()
        self.lib.ora_transport(ctypes.byref(self.c), self.c.mls_order, 0, ctypes.byref(nfix))
        nflag = self.lib.ora_check_pad(ctypes.byref(self.c))
        if nflag > 0:
            self.lib.ora_transport(ctypes.byref(self.c), 1, 1, None)
        return nflag

    def sum_mass(self) -> float:
        self.lib.ora_sum_mass.restype = ctypes.c_double
        return self.lib.ora_sum_mass(ctypes.byref(self.c))

    def body_loads(self, centres, areas):
        nb = len(areas)
        c = np.ascontiguousarray(centres, np.float64).reshape(nb, 3)
        a = np.ascontiguousarray(areas, np.float64)
        out = np.zeros((nb, 6))
        self.lib.ora_body_loads(ctypes.byref(self.c), nb, _p(c), _p(a), _p(out))
        return out

    @staticmethod
    def set_threads(n: int):
        ctypes.CDLL(build_oracle()).ora_set_threads(int(n))


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_library() -> str | None:
    """Path of the widest compiled-reference variant this host can run."""
    flags = _cpu_flags()
    order = []
    if {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= flags:
        order.append("v4")
    if {"avx2", "fma", "bmi2"} <= flags:
        order.append("v3")
    order.append("base")
    for isa in order:
        p = os.path.join(REF_DIR, f"libalebgk_ref_{isa}.so")
        if os.path.exists(p):
            return p
    return None


def ref_cuda_library() -> str | None:
    """Path of the reference built with its own CUDA backend for sm_100a."""
    p = os.path.join(REF_DIR, "libalebgk_refcuda.so")
    return p if os.path.exists(p) else None


class RefCase:
    """A case built and stepped by the reference's own CPU code."""

    def __init__(self, name, Nx=-1, Nv=-1, dt=-1.0, mls_order=2, fixed_body=False,
                 body_scale=1.0, lib_path=None):
        path = lib_path or ref_library()
        if path is None:
            raise FileNotFoundError("oracle/_ref is not built (make -C oracle ref)")
        self.path = path
        L = ctypes.CDLL(path)
        L.ref_create.restype = _vp
        L.ref_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.ref_sum_mass.restype = ctypes.c_double
        L.ref_max_threads.restype = ctypes.c_int
        if hasattr(L, "ref_write_vtk"):
            L.ref_write_vtk.argtypes = [_vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
            L.ref_write_timeseries.argtypes = [_vp, ctypes.c_char_p, ctypes.c_double]
            L.ref_print_step.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        self.L = L
        self.h = _vp(L.ref_create(name.encode(), int(Nx), int(Nv), float(dt), int(mls_order),
                                  int(bool(fixed_body)), float(body_scale)))
        if not self.h.value:
            raise ValueError(f"unknown case {name}")
        d = (ctypes.c_int * 6)()
        L.ref_dims(self.h, d)
        self.N, self.dim, self.Nv, self.gs, self.nbodies, self.mls_order = list(d)
        self._params()

    def _params(self):
        p = np.zeros(24)
        self.L.ref_params(self.h, _p(p))
        keys = ("dt", "tau", "R", "dx", "dy", "dz", "radius", "minDist", "dv", "vmin",
                "vmax", "rho0", "Tw", "xleft", "xright", "ybottom", "ytop", "zfront",
                "zback", "t", "step", "dHS", "tau_variable", "moving")
        self.params = dict(zip(keys, p))
        self.dt = self.params["dt"]

    def cloud(self):
        N = self.N
        xyz = np.zeros((N, 3)); mv = np.zeros((N, 3)); wall = np.zeros((N, 7))
        ints = np.zeros((N, 3), np.int32); nbr = np.zeros((N, MAX_NEIGH), np.int32)
        self.L.ref_get_cloud(self.h, _p(xyz), _p(mv), _p(wall), _p(ints), _p(nbr))
        return dict(xyz=xyz, meshv=mv, wall=wall, boundary=ints[:, 0].copy(),
                    body_id=ints[:, 1].copy(), nnb=ints[:, 2].copy(), nbr=nbr)

    def g(self):
        g = np.zeros((self.N, self.gs))
        self.L.ref_get_g(self.h, _p(g))
        return g

    def gt(self):
        g = np.zeros((self.N, self.gs))
        self.L.ref_get_gt(self.h, _p(g))
        return g

    def macro(self):
        m = np.zeros((self.N, 7))
        self.L.ref_get_macros(self.h, _p(m))
        return m

    def set_g(self, g):
        g = np.ascontiguousarray(g, np.float64)
        self.L.ref_set_g(self.h, _p(g))

    def set_macro(self, m):
        m = np.ascontiguousarray(m, np.float64)
        self.L.ref_set_macros(self.h, _p(m))

    def step(self, n=1):
        self.L.ref_step(self.h, int(n))
        d = (ctypes.c_int * 6)()
        self.L.ref_dims(self.h, d)
        self.N = d[0]
        last = (ctypes.c_int * 2)()
        self.L.ref_last_flags(self.h, last)
        return {"transport_flags": last[0], "mood_fail": last[1]}

    def transport(self):
        return self.L.ref_transport(self.h)

    def sum_mass(self):
        return self.L.ref_sum_mass(self.h)

    # The reference's save-cycle output (Core/Output.hpp) of the case's
    # particles: a VTK frame, diagnostics, a timeseries row (the first call
    # in the process writes the column line) and the step line on stdout.
    def write_vtk(self, outdir, step, time):
        self.L.ref_write_vtk(self.h, str(outdir).encode(), int(step), float(time))

    def diagnostics(self):
        d = np.zeros(6)
        self.L.ref_diagnostics(self.h, _p(d))
        return dict(rho_avg=d[0], KE=d[1], T_avg=d[2], p_avg=d[3], mood_count=int(d[4]),
                    n=int(d[5]))

    def write_timeseries(self, path, t):
        self.L.ref_write_timeseries(self.h, str(path).encode(), float(t))

    def print_step(self, step, t, dt):
        self.L.ref_print_step(self.h, int(step), float(t), float(dt))

    def bodies(self):
        out = np.zeros((max(1, self.nbodies), 32))
        self.L.ref_get_bodies(self.h, _p(out))
        return out[: self.nbodies]

    def set_threads(self, n):
        self.L.ref_set_threads(int(n))

    def cuda_run(self, warmup: int, steps: int) -> float:
        """Steps the case on the reference's own CUDA backend
        (Solver/CudaBackend.cu; needs the library of :func:`ref_cuda_library`):
        upload, ``warmup`` untimed and ``steps`` timed cudaStep calls, then the
        moments come back into this case.  Returns ms per timed step."""
        if not hasattr(self.L, "ref_cuda_run"):
            raise RuntimeError("not the reference CUDA build (oracle/_ref/libalebgk_refcuda.so)")
        ms = ctypes.c_double()
        self.L.ref_cuda_run.argtypes = [_vp, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
        rc = self.L.ref_cuda_run(self.h, int(warmup), int(steps), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError("the reference CUDA backend failed")
        return ms.value

    def checkpoint_save(self, path: str) -> bool:
        """The reference's ckpt::save (Core/Checkpoint.hpp:84-155)."""
        return bool(self.L.ref_checkpoint_save(self.h, path.encode()))

    def checkpoint_load(self, path: str):
        """The reference's ckpt::restore (Core/Checkpoint.hpp:157-236)."""
        step = ctypes.c_long()
        t = ctypes.c_double()
        ok = self.L.ref_checkpoint_load(self.h, path.encode(), ctypes.byref(step),
                                        ctypes.byref(t))
        return bool(ok), step.value, t.value

    def checkpoint_sizes(self):
        out = (ctypes.c_int * 3)()
        self.L.ref_checkpoint_sizes(out)
        return tuple(out)

    def max_threads(self):
        return self.L.ref_max_threads()

    def oracle(self, **kw) -> Oracle:
        """An :class:`Oracle` started from this case's current state."""
        c = self.cloud()
        p = self.params
        return Oracle(dim=self.dim, Nv=self.Nv, dt=self.dt, tau=p["tau"], R=p["R"],
                      dHS=p["dHS"], vmin=p["vmin"], dv=p["dv"], h=p["radius"], g=self.g(),
                      macro=self.macro(), mls_order=kw.pop("mls_order", self.mls_order),
                      **c, **kw)

    def __del__(self):
        try:
            self.L.ref_destroy(self.h)
        except Exception:
            pass
