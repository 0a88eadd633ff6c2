"""B200-native ALE-BGK time step behind the reference's solver-step interface.

Host-side mirror of panchiittp/ALEBGK4Paper's GPU driver API
(Solver/Solver.cpp:67-89): :class:`Case` builds one of the reference's six
lid-driven-cavity clouds on the host (TestCases/TestCases.cpp:56-294), and
:class:`Solver` keeps it on one B200 and advances it with the sm_100a kernels
of ``libalebgk_b200.so`` through the C-ABI of ``include/alebgk.h``.  Method
names follow the reference's ``cuda*`` functions so that code written against
the reference reads the same.  There is no CPU fallback: every call goes
through the CUDA library and fails loudly if it cannot.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi

__all__ = ["Case", "LatticeCase", "Solver", "AlebgkError", "load_library", "read_checkpoint",
           "CASE_NAMES", "diagnostics", "write_vtk_host", "write_timeseries", "format_step",
           "read_fields"]

CASE_NAMES = ("cavity2d", "cavity3d", "cavity2d-square", "cavity2d-circle",
              "cavity3d-sphere", "cavity3d-cube")


class AlebgkError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"alebgk error {code}: {msg}")
        self.code = code


def load_library():
    return _abi.load()


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_abi.c_double_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_abi.c_int_p)


def _check(rc: int, ctx=None):
    if rc != 0:
        lib = _abi.load()
        buf = ctypes.create_string_buffer(512)
        lib.alebgk_last_error(ctx, buf, 512)
        raise AlebgkError(rc, buf.value.decode(errors="replace"))


def read_checkpoint(path: str, N: int | None = None, gstride: int | None = None,
                    dim: int | None = None, nbodies: int | None = None) -> dict:
    """Reads a restart file in the reference's layout (Core/Checkpoint.hpp)
    on the host: header fields plus xyz, meshv, wall, boundary, body_id, g,
    macro, voxel and the body states.  Expected shapes default to the
    file's own."""
    lib = _abi.load()
    h = _abi.CkptHeader()
    _check(lib.alebgk_checkpoint_header(str(path).encode(), ctypes.byref(h)))
    exp = _abi.CkptHeader(N=h.N if N is None else N, gstride=h.gstride if gstride is None
                          else gstride, step=h.step, t=h.t,
                          dim=h.dim if dim is None else dim,
                          nbodies=h.nbodies if nbodies is None else nbodies)
    n, gs, nb = int(exp.N), int(exp.gstride), int(exp.nbodies)
    out = dict(step=int(h.step), t=float(h.t), dim=int(h.dim), N=n, gstride=gs,
               xyz=np.zeros((n, 3)), meshv=np.zeros((n, 3)), wall=np.zeros((n, 7)),
               boundary=np.zeros(n, np.int32), body_id=np.zeros(n, np.int32),
               g=np.zeros((n, gs)), macro=np.zeros((n, 7)), voxel=np.zeros(n, np.int32))
    cl = _abi.Cloud(_dp(out["xyz"]), _dp(out["meshv"]), _dp(out["wall"]), _ip(out["boundary"]),
                    _ip(out["body_id"]), None, None, _dp(out["g"]), _dp(out["macro"]))
    bodies = (_abi.Body * max(1, nb))()
    _check(lib.alebgk_checkpoint_read(str(path).encode(), ctypes.byref(exp), ctypes.byref(cl),
                                      _ip(out["voxel"]), bodies))
    out["bodies"] = np.array([[bodies[b].state[k] for k in range(32)] for b in range(nb)])
    out["body_rotates"] = np.array([bodies[b].rotates for b in range(nb)], np.int32)
    return out


def _diag_dict(d) -> dict:
    return {k: getattr(d, k) for k, _ in _abi.Diag._fields_}


def _diag_struct(d: dict):
    return _abi.Diag(**{k: d[k] for k, _ in _abi.Diag._fields_})


def diagnostics(macro: np.ndarray, boundary: np.ndarray) -> dict:
    """Interior averages of rho, kinetic energy, T, p, the moodFlag count and
    the interior count from host arrays (macro N x 7, boundary N), in
    particle order as computeDiagnostics (Core/Output.hpp:66-85)."""
    lib = _abi.load()
    m = np.ascontiguousarray(macro, np.float64)
    b = np.ascontiguousarray(boundary, np.int32)
    d = _abi.Diag()
    _check(lib.alebgk_diagnostics_host(int(m.shape[0]), _dp(m), _ip(b), ctypes.byref(d)))
    return _diag_dict(d)


def write_vtk_host(path: str, xyz: np.ndarray, macro: np.ndarray, boundary: np.ndarray,
                   Nv: int, time: float = 0.0):
    """The reference's ASCII VTK frame (Core/Output.hpp:17-51) of host arrays."""
    lib = _abi.load()
    x = np.ascontiguousarray(xyz, np.float64)
    m = np.ascontiguousarray(macro, np.float64)
    b = np.ascontiguousarray(boundary, np.int32)
    _check(lib.alebgk_vtk_write_host(str(path).encode(), int(x.shape[0]), _dp(x), _dp(m), _ip(b),
                                     int(Nv), float(time)))


def write_timeseries(path: str, t: float, diag: dict, header: bool = False):
    """One timeseries.csv row (Core/Output.hpp:91-106); header=True truncates
    the file and writes the column line first."""
    d = _diag_struct(diag)
    _check(_abi.load().alebgk_write_timeseries(str(path).encode(), float(t), ctypes.byref(d),
                                               int(bool(header))))


def format_step(step: int, t: float, dt: float, diag: dict) -> str:
    """The reference's step line (printStep, Core/Output.hpp:111-115)."""
    buf = ctypes.create_string_buffer(256)
    d = _diag_struct(diag)
    _check(_abi.load().alebgk_format_step(buf, 256, int(step), float(t), float(dt),
                                          ctypes.byref(d)))
    return buf.value.decode()


def read_fields(path: str) -> dict:
    """Reads a binary field dump (alebgk_write_fields): step, t, dim and the
    xyz (N x 3), macro (N x 7) and boundary (N) arrays."""
    lib = _abi.load()
    h = _abi.FieldsHeader()
    _check(lib.alebgk_read_fields(str(path).encode(), ctypes.byref(h), None, None, None))
    n = int(h.N)
    out = dict(step=int(h.step), t=float(h.t), dim=int(h.dim), N=n, xyz=np.zeros((n, 3)),
               macro=np.zeros((n, 7)), boundary=np.zeros(n, np.int32))
    _check(lib.alebgk_read_fields(str(path).encode(), ctypes.byref(h), _dp(out["xyz"]),
                                  _dp(out["macro"]), _ip(out["boundary"])))
    return out


class Case:
    """A case cloud built on the host, as TestCases/main.cpp:193-345 builds it.

    Arrays (numpy, owned by this object): ``xyz`` (N,3), ``meshv`` (N,3),
    ``wall`` (N,7), ``boundary`` (N,), ``body_id`` (N,), ``nnb`` (N,),
    ``nbr`` (N,128), ``g`` (N,gstride) FP64, ``macro`` (N,7).
    """

    def __init__(self, name: str, Nx: int = -1, Nv: int = -1, dt: float = -1.0,
                 mls_order: int = 2, fixed_body: bool = False, body_scale: float = 1.0,
                 lid_speed: float = -1.0, rho0: float = -1.0, tau: float = -1.0):
        lib = _abi.load()
        h = ctypes.c_void_p()
        _check(lib.alebgk_case_build_ex(name.encode(), int(Nx), int(Nv), float(dt),
                                        int(mls_order), int(bool(fixed_body)),
                                        float(body_scale), float(lid_speed), float(rho0),
                                        float(tau), ctypes.byref(h)))
        try:
            info = np.zeros(8, np.int32)
            prm = np.zeros(24)
            _check(lib.alebgk_case_info(h, _ip(info), _dp(prm)))
            view = _abi.Cloud()
            _check(lib.alebgk_case_view(h, ctypes.byref(view)))
            N, gs = int(info[0]), int(info[3])
            self.name = name
            self.N, self.dim, self.Nv, self.gstride = N, int(info[1]), int(info[2]), gs
            self.nbodies, self.mls_order, self.Nx = int(info[4]), int(info[5]), int(info[6])
            self.moving_bodies = bool(info[7])
            keys = ("dt", "tau", "R", "dx", "dy", "dz", "radius", "minDist", "dv",
                    "vmin", "vmax", "rho0", "Tw", "xleft", "xright", "ybottom", "ytop",
                    "zfront", "zback", "dt_requested", "tfinal", "dHS", "lid_speed",
                    "save_every")
            self.params = {k: float(v) for k, v in zip(keys, prm)}
            self.dt = self.params["dt"]

            def arr(ptr, n, dtype, shape):
                return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).reshape(shape)

            self.xyz = arr(view.xyz, 3 * N, np.float64, (N, 3))
            self.meshv = arr(view.meshv, 3 * N, np.float64, (N, 3))
            self.wall = arr(view.wall, 7 * N, np.float64, (N, 7))
            self.boundary = arr(view.boundary, N, np.int32, (N,))
            self.body_id = arr(view.body_id, N, np.int32, (N,))
            self.nnb = arr(view.nnb, N, np.int32, (N,))
            self.nbr = arr(view.nbr, N * _abi.MAX_NEIGH, np.int32, (N, _abi.MAX_NEIGH))
            self.g = arr(view.g, N * gs, np.float64, (N, gs))
            self.macro = arr(view.macro, 7 * N, np.float64, (N, 7))
            bodies = np.zeros(32 * max(1, self.nbodies))
            _check(lib.alebgk_case_bodies(h, _dp(bodies)))
            self.bodies = bodies.reshape(-1, 32)[: self.nbodies].copy()
            kind = np.zeros(max(1, self.nbodies), np.int32)
            rot = np.zeros(max(1, self.nbodies), np.int32)
            size = np.zeros(max(1, self.nbodies))
            _check(lib.alebgk_case_body_shapes(h, _ip(kind), _ip(rot), _dp(size)))
            self.body_kind = kind[: self.nbodies].copy()
            self.body_rotates = rot[: self.nbodies].copy()
            self.body_size = size[: self.nbodies].copy()
        finally:
            lib.alebgk_case_free(h)

    def config(self, precision: int = 32, device: int = 0, transport: int = 0,
               particle: int = 0) -> _abi.Config:
        cfg = _abi.Config()
        cfg.transport = transport
        cfg.particle = particle
        cfg.dim, cfg.N, cfg.Nv = self.dim, self.N, self.Nv
        cfg.mls_order, cfg.precision, cfg.limiter = self.mls_order, precision, 2
        cfg.tau_variable, cfg.device = 0, device
        cfg.R, cfg.tau, cfg.dHS = self.params["R"], self.params["tau"], self.params["dHS"]
        cfg.vmin, cfg.dv, cfg.radius = self.params["vmin"], self.params["dv"], self.params["radius"]
        return cfg

    def cloud(self) -> _abi.Cloud:
        """A C-ABI view of this case's arrays (kept alive by this object); g
        is NULL once a particle-set change kept the distribution on the
        device (``Solver.refresh_geometry``)."""
        self._keep = [None if a is None else np.ascontiguousarray(a) for a in
                      (self.xyz, self.meshv, self.wall, self.boundary, self.body_id,
                       self.nnb, self.nbr, self.g, self.macro)]
        xyz, mv, wall, b, bid, nnb, nbr, g, mac = self._keep
        return _abi.Cloud(_dp(xyz), _dp(mv), _dp(wall), _ip(b), _ip(bid), _ip(nnb),
                          _ip(nbr), None if g is None else _dp(g), _dp(mac))


class LatticeCase:
    """A case whose set-up runs on the device.

    It carries the case parameters (``alebgk_lattice_info_ex``) and the
    bodies' descriptions (``alebgk_lattice_bodies``); the lattice, wall
    state, body embedding, neighbour lists and rest state are built on the
    GPU when a :class:`Solver` takes it (``alebgk_upload_lattice_ex``),
    bitwise equal to what :class:`Case` builds on the host.  Same arguments
    as :class:`Case`; for a case with bodies the particle count after the
    embedding comes from a device set-up on ``device``, and the host arrays
    a moving-body run manages (positions, flags, wall state, neighbours) are
    fetched from it.
    """

    def __init__(self, name: str, Nx: int = -1, Nv: int = -1, dt: float = -1.0,
                 mls_order: int = 2, lid_speed: float = -1.0, rho0: float = -1.0,
                 tau: float = -1.0, fixed_body: bool = False, body_scale: float = 1.0,
                 device: int = 0):
        lib = _abi.load()
        self._args = (name.encode(), int(Nx), int(Nv), float(dt), int(mls_order),
                      int(bool(fixed_body)), float(body_scale), float(lid_speed), float(rho0),
                      float(tau))
        info = np.zeros(8, np.int32)
        prm = np.zeros(24)
        _check(lib.alebgk_lattice_info_ex(*self._args, int(device), _ip(info), _dp(prm)))
        self.name = name
        self.N, self.dim, self.Nv, self.gstride = int(info[0]), int(info[1]), int(info[2]), \
            int(info[3])
        self.nbodies, self.mls_order, self.Nx = int(info[4]), int(info[5]), int(info[6])
        self.moving_bodies = bool(info[7])
        keys = ("dt", "tau", "R", "dx", "dy", "dz", "radius", "minDist", "dv",
                "vmin", "vmax", "rho0", "Tw", "xleft", "xright", "ybottom", "ytop",
                "zfront", "zback", "dt_requested", "tfinal", "dHS", "lid_speed",
                "save_every")
        self.params = {k: float(v) for k, v in zip(keys, prm)}
        self.dt = self.params["dt"]
        nb = max(1, self.nbodies)
        st, kind = np.zeros(32 * nb), np.zeros(nb, np.int32)
        rot, size = np.zeros(nb, np.int32), np.zeros(nb)
        n = ctypes.c_int()
        _check(lib.alebgk_lattice_bodies(*self._args[:7], ctypes.byref(n), _dp(st), _ip(kind),
                                         _ip(rot), _dp(size)))
        self.bodies = st.reshape(-1, 32)[: self.nbodies].copy()
        self.body_kind = kind[: self.nbodies].copy()
        self.body_rotates = rot[: self.nbodies].copy()
        self.body_size = size[: self.nbodies].copy()
        self._xyz = None
        # host distribution and macros: none until a cloud-management change
        # of a moving-body run reads them back (then uploads go through them)
        self.g = self.macro = None
        if self.nbodies:
            out = self.build_on_device(device)
            self.meshv = np.zeros((self.N, 3))
            for k in ("wall", "boundary", "body_id", "nnb", "nbr"):
                setattr(self, k, out[k])

    config = Case.config

    def cloud(self) -> _abi.Cloud:
        """A C-ABI view of the host arrays (geometry; g and macro only once a
        cloud-management change has read them back)."""
        self._keep = [None if a is None else np.ascontiguousarray(a) for a in
                      (self.xyz, self.meshv, self.wall, self.boundary, self.body_id,
                       self.nnb, self.nbr, self.g, self.macro)]
        xyz, mv, wall, b, bid, nnb, nbr, g, mac = self._keep
        return _abi.Cloud(_dp(xyz), _dp(mv), _dp(wall), _ip(b), _ip(bid), _ip(nnb), _ip(nbr),
                          None if g is None else _dp(g), None if mac is None else _dp(mac))

    @property
    def xyz(self) -> np.ndarray:
        """Particle positions (N, 3), from the device set-up."""
        if self._xyz is None:
            self._xyz = self.build_on_device()["xyz"]
        return self._xyz

    @xyz.setter
    def xyz(self, value: np.ndarray):
        self._xyz = value

    def build_on_device(self, device: int = 0) -> dict:
        """The device-built arrays: xyz, wall, boundary, body_id, nnb, nbr."""
        lib = _abi.load()
        N = self.N
        out = dict(xyz=np.zeros((N, 3)), wall=np.zeros((N, 7)),
                   boundary=np.zeros(N, np.int32), body_id=np.zeros(N, np.int32),
                   nnb=np.zeros(N, np.int32), nbr=np.zeros((N, _abi.MAX_NEIGH), np.int32))
        _check(lib.alebgk_lattice_build_device_ex(*self._args, int(device), _dp(out["xyz"]),
                                                  _dp(out["wall"]), _ip(out["boundary"]),
                                                  _ip(out["body_id"]), _ip(out["nnb"]),
                                                  _ip(out["nbr"])))
        self._xyz = out["xyz"]
        return out


class Solver:
    """One device-resident cloud advanced by the B200 step.

    Mirrors the reference's CUDA driver API (Solver/Solver.cpp:67-89):
    construction is ``cudaUploadCloud``; ``cudaStep``, ``cudaDownloadMoments``,
    ``cudaDownloadFull``, ``cudaTotalMass``, ``cudaLimiterCounts``,
    ``cudaMlsCounts``, ``cudaMassBudget``, ``cudaWallMomentum`` and
    ``cudaFreeCloud`` keep the reference's names and meaning.
    """

    def __init__(self, case: Case, precision: int = 32, device: int = 0,
                 dt: float | None = None, config: _abi.Config | None = None,
                 transport: int = 0, particle: int = 0):
        self.lib = _abi.load()
        self.case = case
        self.N, self.gstride, self.dim = case.N, case.gstride, case.dim
        self.precision = precision
        self.dt = float(dt if dt is not None else case.dt)
        cfg = config if config is not None else case.config(precision, device, transport,
                                                              particle)
        self.cfg = cfg
        h = ctypes.c_void_p()
        _check(self.lib.alebgk_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.ctx = h
        self.cudaUploadCloud(case)

    # -- reference-named API ------------------------------------------------
    def cudaUploadCloud(self, case: Case):
        if isinstance(case, LatticeCase) and case.g is None and \
                not getattr(case, "_managed", False):
            _check(self.lib.alebgk_upload_lattice_ex(self.ctx, *case._args), self.ctx)
            return
        cl = case.cloud()
        _check(self.lib.alebgk_upload(self.ctx, ctypes.byref(cl), self.dt), self.ctx)

    def cudaStep(self, nsteps: int = 1):
        _check(self.lib.alebgk_step(self.ctx, int(nsteps)), self.ctx)

    step = cudaStep

    def sync(self):
        _check(self.lib.alebgk_sync(self.ctx), self.ctx)

    def cudaDownloadMoments(self, out: np.ndarray | None = None) -> np.ndarray:
        m = out if out is not None else np.zeros((self.N, 7))
        _check(self.lib.alebgk_download_moments(self.ctx, _dp(m)), self.ctx)
        return m

    def cudaDownloadFull(self):
        g = np.zeros((self.N, self.gstride))
        m = np.zeros((self.N, 7))
        _check(self.lib.alebgk_download_full(self.ctx, _dp(g), _dp(m)), self.ctx)
        return g, m

    def counters(self) -> dict:
        c = _abi.Counters()
        _check(self.lib.alebgk_get_counters(self.ctx, ctypes.byref(c)), self.ctx)
        return {k: getattr(c, k) for k, _ in _abi.Counters._fields_}

    def cudaLimiterCounts(self):
        c = self.counters()
        return c["positivity_fixes"], c["transport_flags"]

    def cudaMlsCounts(self):
        c = self.counters()
        return c["mls_degenerate"], 0

    def cudaMassBudget(self):
        c = self.counters()
        return c["mass_after_transport"] * c["mass_scale"], c["mass_end"]

    def cudaTotalMass(self) -> float:
        v = ctypes.c_double()
        _check(self.lib.alebgk_total_mass(self.ctx, ctypes.byref(v)), self.ctx)
        return v.value

    def cudaWallMomentum(self) -> np.ndarray:
        d = np.zeros(self.N)
        _check(self.lib.alebgk_wall_momentum(self.ctx, _dp(d)), self.ctx)
        return d

    def body_loads(self, centres: np.ndarray, areas: np.ndarray) -> np.ndarray:
        nb = len(areas)
        c = np.ascontiguousarray(centres, np.float64).reshape(nb, 3)
        a = np.ascontiguousarray(areas, np.float64)
        out = np.zeros((nb, 6))
        _check(self.lib.alebgk_body_loads(self.ctx, nb, _dp(c), _dp(a), _dp(out)), self.ctx)
        return out

    def body_loads_noalloc(self, centres: np.ndarray, areas: np.ndarray) -> np.ndarray:
        """Same loads as :meth:`body_loads` from a fixed device scratch, with no
        device allocation (at most ``_abi.NOALLOC_MAX_BODIES`` bodies; calls that
        overlap on one device race on the shared scratch)."""
        nb = len(areas)
        c = np.ascontiguousarray(centres, np.float64).reshape(nb, 3)
        a = np.ascontiguousarray(areas, np.float64)
        out = np.zeros((nb, 6))
        _check(self.lib.alebgk_body_loads_noalloc(self.ctx, nb, _dp(c), _dp(a), _dp(out)),
               self.ctx)
        return out

    def body_step(self, state: np.ndarray | None = None, dt: float | None = None) -> np.ndarray:
        """One Heun Newton-Euler step of the case's bodies after a completed
        step (moveRigidBodies, RigidBody/BodyDynamics.cpp:352-638).  ``state``
        (nbodies x 32, the layout of :attr:`Case.bodies`) defaults to the
        case's; the updated state is returned.  The surface particles move,
        so the next :meth:`cudaStep` needs the cloud uploaded again."""
        c = self.case
        st = np.ascontiguousarray(c.bodies if state is None else state, np.float64)
        nb = st.shape[0]
        arr = (_abi.Body * nb)()
        for b in range(nb):
            arr[b].kind = int(c.body_kind[b])
            arr[b].rotates = int(c.body_rotates[b])
            arr[b].size = float(c.body_size[b])
            for k in range(32):
                arr[b].state[k] = float(st[b, k])
        p = c.params
        box = np.array([p["xleft"], p["xright"], p["ybottom"], p["ytop"], p["zfront"],
                        p["zback"]])
        _check(self.lib.alebgk_body_step(self.ctx, nb, arr, _dp(box), float(p["dx"]),
                                         float(self.dt if dt is None else dt)), self.ctx)
        return np.array([[arr[b].state[k] for k in range(32)] for b in range(nb)])

    def neighbour_grid(self):
        """(grid, boxes) of the case's voxel binning (ParticleGeneration.cpp
        box sizes 3 dx, 3 dy, 3 dz; NeighbourSearch.cpp:17-99)."""
        import math
        p = self.case.params
        d3 = self.case.dim == 3
        hx, hy = 3.0 * p["dx"], 3.0 * p["dy"]
        hz = 3.0 * p["dz"] if d3 else 1.0
        nx = int(math.ceil((p["xright"] - p["xleft"]) / hx)) + 1
        ny = int(math.ceil((p["ytop"] - p["ybottom"]) / hy)) + 1
        nz = int(math.ceil((p["zback"] - p["zfront"]) / hz)) + 1 if d3 else 1
        grid = np.array([p["xleft"], p["ybottom"], p["zfront"], hx, hy, hz, p["radius"]])
        return grid, np.array([nx, ny, nz], np.int32)

    def rebuild_neighbours(self):
        """Neighbour lists (nnb, nbr) of the device's current positions,
        built on the device (updateVoxelsAndNeighbours,
        NeighbourSearch.cpp:17-99)."""
        grid, boxes = self.neighbour_grid()
        nnb = np.zeros(self.N, np.int32)
        nbr = np.zeros((self.N, _abi.MAX_NEIGH), np.int32)
        _check(self.lib.alebgk_neighbours_device(self.ctx, _dp(grid), _ip(boxes), _ip(nnb),
                                                 _ip(nbr)), self.ctx)
        return nnb, nbr

    def refresh_geometry(self, bodies: np.ndarray | None = None, manage: bool = True,
                         device_state: bool = True):
        """Uploads the cloud again after :meth:`body_step` moved the surface:
        positions, mesh velocities and wall state as the device holds them.
        With ``manage`` (and bodies in the case) the reference's cloud
        management runs first -- remove, merge, refill and the neighbour
        rebuilds of Solver.cpp:381-395 (:func:`alebgk4paper_b200.cloud.
        manage_cloud`), for the bodies at ``bodies`` (nbodies x 32, default
        the case's); otherwise only the neighbour lists are rebuilt on the
        device.  While the particle set stays the same (the usual step) the
        distribution never leaves the device (``alebgk_upload_geometry``);
        when it changes, the state is read back, managed and uploaded, and
        the context is rebuilt for the new particle count: with
        ``device_state`` the distribution never leaves the device then either
        (the management returns a row plan, ``alebgk_rows_build`` builds the
        new rows from the old context and ``alebgk_upload_rows`` installs them
        after a geometry-only upload); without it the state is read back,
        managed on the host and uploaded.  Both give bitwise the same state.
        Returns the cloud management counts (removed, merged, added)."""
        from .cloud import manage_cloud
        c = self.case
        xyz, mv, wall = self.download_geometry()
        c.xyz, c.meshv, c.wall = xyz, mv, wall
        counts = (0, 0, 0)
        if manage and getattr(c, "nbodies", 0):
            st = c.bodies if bodies is None else bodies
            geo = dict(xyz=xyz, meshv=mv, wall=wall, boundary=c.boundary, body_id=c.body_id)
            out, counts, need = manage_cloud(c, geo, st, self.cfg.device, decide_only=True)
            if need and device_state:
                return self._refresh_device_state(c, geo, st)
            if need:
                g, macro = self.cudaDownloadFull()
                geo.update(g=g, macro=macro)
                out, counts, _ = manage_cloud(c, geo, st, self.cfg.device)
                c.xyz, c.meshv, c.wall = out["xyz"], out["meshv"], out["wall"]
                c.boundary, c.body_id = out["boundary"], out["body_id"]
                c.nnb, c.nbr, c.g, c.macro = out["nnb"], out["nbr"], out["g"], out["macro"]
                if len(c.xyz) != self.N:
                    c.N = self.N = len(c.xyz)
                    self.lib.alebgk_destroy(self.ctx)
                    self.cfg.N = self.N
                    h = ctypes.c_void_p()
                    _check(self.lib.alebgk_create(ctypes.byref(self.cfg), ctypes.byref(h)))
                    self.ctx = h
                self.cudaUploadCloud(c)
                return counts
            c.nnb, c.nbr = out["nnb"], out["nbr"]
        else:
            c.nnb, c.nbr = self.rebuild_neighbours()
        cl = c.cloud()
        _check(self.lib.alebgk_upload_geometry(self.ctx, ctypes.byref(cl), self.dt), self.ctx)
        return counts

    def _refresh_device_state(self, c, geo, st):
        """The particle-set change of :meth:`refresh_geometry` with the
        distribution kept on the device."""
        from .cloud import manage_cloud
        geo.update(macro=self.cudaDownloadMoments())
        out, counts, _ = manage_cloud(c, geo, st, self.cfg.device, plan=True)
        a, b, fresh = out["plan"]
        fresh = np.ascontiguousarray(fresh, np.float64)
        rows = ctypes.c_void_p()
        _check(self.lib.alebgk_rows_build(self.ctx, len(a), _ip(a), _ip(b), len(fresh),
                                          _dp(fresh) if len(fresh) else None,
                                          ctypes.byref(rows)), self.ctx)
        try:
            c.xyz, c.meshv, c.wall = out["xyz"], out["meshv"], out["wall"]
            c.boundary, c.body_id = out["boundary"], out["body_id"]
            c.nnb, c.nbr, c.macro = out["nnb"], out["nbr"], out["macro"]
            c.g = None
            c._managed = True
            if len(c.xyz) != self.N:
                c.N = self.N = len(c.xyz)
                self.lib.alebgk_destroy(self.ctx)
                self.cfg.N = self.N
                h = ctypes.c_void_p()
                _check(self.lib.alebgk_create(ctypes.byref(self.cfg), ctypes.byref(h)))
                self.ctx = h
            keep = [np.ascontiguousarray(x) for x in (c.xyz, c.meshv, c.wall, c.boundary,
                                                        c.body_id, c.nnb, c.nbr)]
            xyz, mv, wall, bd, bid, nnb, nbr = keep
            cl = _abi.Cloud(_dp(xyz), _dp(mv), _dp(wall), _ip(bd), _ip(bid), _ip(nnb), _ip(nbr),
                            None, None)
            _check(self.lib.alebgk_upload(self.ctx, ctypes.byref(cl), self.dt), self.ctx)
            mac = np.ascontiguousarray(c.macro, np.float64)
            r, rows = rows, None
            _check(self.lib.alebgk_upload_rows(self.ctx, r, _dp(mac)), self.ctx)
        finally:
            if rows is not None and rows.value:
                self.lib.alebgk_rows_free(rows)
        return counts

    def write_vtk(self, outdir: str, step: int, time: float):
        """The reference's VTK frame of the current state into
        outdir/output_%06d.vtk (Core/Output.hpp:17-51)."""
        _check(self.lib.alebgk_write_vtk(self.ctx, str(outdir).encode(), int(step), float(time)),
               self.ctx)

    def diagnostics(self) -> dict:
        """Interior averages of the current state (Core/Output.hpp:66-85)."""
        d = _abi.Diag()
        _check(self.lib.alebgk_diagnostics(self.ctx, ctypes.byref(d)), self.ctx)
        return _diag_dict(d)

    def write_fields(self, path: str, step: int = 0, t: float = 0.0):
        """Binary field dump of the current state at full precision."""
        _check(self.lib.alebgk_write_fields(self.ctx, str(path).encode(), int(step), float(t)),
               self.ctx)

    def checkpoint_save(self, path: str, step: int = 0, t: float = 0.0,
                        bodies: np.ndarray | None = None, voxel: np.ndarray | None = None):
        """Writes a restart file in the reference's layout (Core/Checkpoint.hpp)
        from the device state; ``bodies`` (nbodies x 32) defaults to the
        case's."""
        c = self.case
        st = np.ascontiguousarray(c.bodies if bodies is None else bodies, np.float64)
        nb = st.shape[0]
        arr = (_abi.Body * max(1, nb))()
        for b in range(nb):
            arr[b].kind = int(c.body_kind[b])
            arr[b].rotates = int(c.body_rotates[b])
            arr[b].size = float(c.body_size[b])
            for k in range(32):
                arr[b].state[k] = float(st[b, k])
        vg = np.array([c.params["vmin"], c.params["vmax"], c.params["dv"]])
        vox = None if voxel is None else np.ascontiguousarray(voxel, np.int32)
        _check(self.lib.alebgk_checkpoint_save(self.ctx, str(path).encode(), int(step),
                                               float(t), _dp(vg),
                                               None if vox is None else _ip(vox), nb, arr),
               self.ctx)

    def checkpoint_restore(self, path: str) -> dict:
        """Reads a restart file of this cloud's shape and continues from it:
        distribution and macros go to the device; if the file's geometry
        (positions, mesh velocity, wall state) differs from the current one,
        the cloud is uploaded again with it (neighbour lists kept).  Returns
        the file's contents (step, t, bodies, ...)."""
        c = self.case
        d = read_checkpoint(path, N=self.N, gstride=self.gstride, dim=self.dim,
                            nbodies=c.nbodies)
        xyz, mv, wall = self.download_geometry()
        if (np.array_equal(xyz, d["xyz"]) and np.array_equal(mv, d["meshv"])
                and np.array_equal(wall, d["wall"])):
            g = np.ascontiguousarray(d["g"])
            m = np.ascontiguousarray(d["macro"])
            _check(self.lib.alebgk_upload_state(self.ctx, _dp(g), _dp(m)), self.ctx)
        else:
            c.xyz, c.meshv, c.wall = d["xyz"], d["meshv"], d["wall"]
            c.g, c.macro = d["g"], d["macro"]
            self.cudaUploadCloud(c)
        return d

    def set_launch(self, transport_threads: int, particle_warps: int):
        _check(self.lib.alebgk_set_launch(self.ctx, int(transport_threads), int(particle_warps)),
               self.ctx)

    def set_march_width(self, velocities_per_lane: int):
        """Velocities per lane of the lattice march (2: packed FMAs, or 1)."""
        _check(self.lib.alebgk_set_march_width(self.ctx, int(velocities_per_lane)), self.ctx)

    def set_residual_speed(self, speed: float):
        """Speed scale of the residual's momentum terms (0: thermal speed)."""
        _check(self.lib.alebgk_set_residual_speed(self.ctx, float(speed)), self.ctx)

    def set_nad_floor(self, rel: float):
        """Relative rounding floor of the FP32 NAD screen (default 64 * 2^-24)."""
        _check(self.lib.alebgk_set_nad_floor(self.ctx, float(rel)), self.ctx)

    def get_launch(self):
        t = ctypes.c_int()
        w = ctypes.c_int()
        _check(self.lib.alebgk_get_launch(self.ctx, ctypes.byref(t), ctypes.byref(w)), self.ctx)
        return t.value, w.value

    def autotune(self, steps: int = 3) -> float:
        """Keeps the fastest launch shape; returns its ms per step."""
        ms = ctypes.c_float()
        _check(self.lib.alebgk_autotune(self.ctx, int(steps), ctypes.byref(ms)), self.ctx)
        return ms.value

    def residual(self) -> float:
        """Steady residual of the last step (relative change of the conserved
        moments over the interior particles)."""
        r = ctypes.c_double()
        _check(self.lib.alebgk_residual(self.ctx, ctypes.byref(r)), self.ctx)
        return r.value

    def residual_interval(self) -> float:
        """Mean steady residual per step since the previous call (-1 on the
        first call, which only takes the snapshot)."""
        r = ctypes.c_double()
        _check(self.lib.alebgk_residual_interval(self.ctx, ctypes.byref(r)), self.ctx)
        return r.value

    def download_geometry(self):
        """(xyz N x 3, meshv N x 3, wall N x 7) as stored on the device."""
        xyz = np.zeros((self.N, 3))
        mv = np.zeros((self.N, 3))
        wall = np.zeros((self.N, 7))
        _check(self.lib.alebgk_download_geometry(self.ctx, _dp(xyz), _dp(mv), _dp(wall)),
               self.ctx)
        return xyz, mv, wall

    def cudaFreeCloud(self):
        if getattr(self, "ctx", None):
            self.lib.alebgk_destroy(self.ctx)
            self.ctx = None

    close = cudaFreeCloud

    def __del__(self):
        try:
            self.cudaFreeCloud()
        except Exception:
            pass
