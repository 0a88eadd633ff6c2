"""Cloud management around moving bodies (``alebgk_manage_cloud``): the
remove / merge / refill block of the reference's moving-body step
(RigidBody/CloudManagement.cpp:17-275, Solver.cpp:381-395) with its
all-particle tests and neighbour rebuilds on the GPU."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from . import _check, _dp, _ip

__all__ = ["manage_cloud"]


def _params(case):
    p = case.params
    d3 = case.dim == 3
    hx, hy = 3.0 * p["dx"], 3.0 * p["dy"]
    hz = 3.0 * p["dz"] if d3 else 1.0
    nx = int(math.ceil((p["xright"] - p["xleft"]) / hx)) + 1
    ny = int(math.ceil((p["ytop"] - p["ybottom"]) / hy)) + 1
    nz = int(math.ceil((p["zback"] - p["zfront"]) / hz)) + 1 if d3 else 1
    prm = np.array([p["dx"], p["minDist"], p["radius"], p["xleft"], p["xright"], p["ybottom"],
                    p["ytop"], p["zfront"], p["zback"], p["vmin"], p["dv"], p["R"], hx, hy, hz])
    iprm = np.array([case.dim, case.Nv, nx, ny, nz], np.int32)
    return prm, iprm


def manage_cloud(case, cloud: dict, bodies_state: np.ndarray, device: int = 0,
                 decide_only: bool = False, plan: bool = False):
    """Runs the cloud management on a host cloud (dict with xyz, meshv, wall,
    boundary, body_id, g, macro) whose bodies are at ``bodies_state``
    (nbodies x 32, the layout of ``Case.bodies``).  Returns (managed cloud
    dict with nnb and nbr, (removed, merged, added), need_state).  With
    ``decide_only`` g and macro are not passed: the call stops with
    need_state True as soon as the particle set would change, and otherwise
    returns the unchanged cloud with rebuilt neighbour lists.  With ``plan``
    the cloud carries macro but no g: the distribution stays with the caller
    (on the device) and the result's "plan" is (a, b, fresh), the origin of
    every row (``alebgk_managed_plan``)."""
    lib = _abi.load()
    prm, iprm = _params(case)
    st = np.ascontiguousarray(bodies_state, np.float64).reshape(-1, 32)
    nb = st.shape[0]
    arr = (_abi.Body * max(nb, 1))()
    for b in range(nb):
        arr[b].kind = int(case.body_kind[b])
        arr[b].rotates = int(case.body_rotates[b])
        arr[b].size = float(case.body_size[b])
        for k in range(32):
            arr[b].state[k] = float(st[b, k])
    names = [("xyz", np.float64), ("meshv", np.float64), ("wall", np.float64),
             ("boundary", np.int32), ("body_id", np.int32)]
    if not decide_only:
        names += ([] if plan else [("g", np.float64)]) + [("macro", np.float64)]
    keep = {k: np.ascontiguousarray(cloud[k], dt) for k, dt in names}
    N = keep["xyz"].shape[0]
    gs = int(case.gstride)
    dummy = np.zeros(1, np.int32)
    none = ctypes.POINTER(ctypes.c_double)()
    cl = _abi.Cloud(_dp(keep["xyz"]), _dp(keep["meshv"]), _dp(keep["wall"]),
                    _ip(keep["boundary"]), _ip(keep["body_id"]), _ip(dummy), _ip(dummy),
                    none if decide_only or plan else _dp(keep["g"]),
                    none if decide_only else _dp(keep["macro"]))
    h = ctypes.c_void_p()
    _check(lib.alebgk_manage_cloud(int(device), _dp(prm), _ip(iprm), nb, arr, N, gs,
                                   ctypes.byref(cl), ctypes.byref(h)))
    try:
        info = np.zeros(5, np.int32)
        _check(lib.alebgk_managed_info(h, _ip(info)))
        counts = (int(info[1]), int(info[2]), int(info[3]))
        if info[4]:
            return None, counts, True
        n = int(info[0])
        view = _abi.Cloud()
        _check(lib.alebgk_managed_cloud(h, ctypes.byref(view)))

        def take(ptr, count, dtype, shape):
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype).reshape(shape)

        out = dict(xyz=take(view.xyz, 3 * n, np.float64, (n, 3)),
                   meshv=take(view.meshv, 3 * n, np.float64, (n, 3)),
                   wall=take(view.wall, 7 * n, np.float64, (n, 7)),
                   boundary=take(view.boundary, n, np.int32, (n,)),
                   body_id=take(view.body_id, n, np.int32, (n,)),
                   nnb=take(view.nnb, n, np.int32, (n,)),
                   nbr=take(view.nbr, n * _abi.MAX_NEIGH, np.int32, (n, _abi.MAX_NEIGH)),
                   g=None if decide_only or plan else take(view.g, n * gs, np.float64, (n, gs)),
                   macro=None if decide_only else take(view.macro, 7 * n, np.float64, (n, 7)))
        if plan:
            a, b = np.zeros(n, np.int32), np.zeros(n, np.int32)
            fresh = np.zeros((max(1, counts[2]), gs))
            _check(lib.alebgk_managed_plan(h, _ip(a), _ip(b), _dp(fresh)))
            out["plan"] = (a, b, fresh[: counts[2]])
        return out, counts, False
    finally:
        lib.alebgk_managed_free(h)
