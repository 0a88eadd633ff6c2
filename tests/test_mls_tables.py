"""Known answers of the MLS transport tables (alebgk_coeff_build, the FP64
coefficients every device transport applies): the reconstruction at a
particle's foot point reproduces every polynomial of the fit's order
(MLSTransport.cpp:129-186 fits the basis of MLSBasis.hpp:158-195), so the
coefficients applied to such a field sampled at the neighbours give the
field at the foot point."""
import ctypes

import numpy as np
import pytest

import alebgk4paper_b200 as ab
from alebgk4paper_b200 import _abi


def _tables(case):
    lib = _abi.load()
    cfg = case.config(64)
    cl = case.cloud()
    h = ctypes.c_void_p()
    assert lib.alebgk_coeff_build(ctypes.byref(cfg), ctypes.byref(cl), case.dt,
                                  ctypes.byref(h)) == 0
    try:
        info = np.zeros(5, np.int32)
        lib.alebgk_coeff_info(h, info.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        ncls, S, V = int(info[0]), int(info[1]), int(info[2])
        cls = np.zeros(case.N, np.int32)
        nslot = np.zeros(case.N, np.int32)
        slots = np.zeros(case.N * S, np.int32)
        coef = np.zeros(ncls * S * V)
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        lib.alebgk_coeff_get(h, ip(cls), ip(nslot), ip(slots),
                             coef.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    finally:
        lib.alebgk_coeff_free(h)
    return cls, nslot, slots.reshape(case.N, S), coef.reshape(ncls, S, V), V


def _velocities(case, V):
    Nv, dv, vmin = case.Nv, case.params["dv"], case.params["vmin"]
    k = np.arange(V)
    v = np.zeros((V, 3))
    v[:, 0] = vmin + (k % Nv) * dv
    v[:, 1] = vmin + (k // Nv % Nv) * dv
    if case.dim == 3:
        v[:, 2] = vmin + (k // (Nv * Nv)) * dv
    return v


@pytest.mark.parametrize("name,Nx,Nv,order", [("cavity3d", 8, 6, 2), ("cavity3d", 8, 6, 1),
                                              ("cavity2d", 12, 8, 2), ("cavity2d", 12, 8, 1)])
def test_tables_reproduce_polynomials_of_the_fit_order(name, Nx, Nv, order):
    c = ab.Case(name, Nx, Nv, -1.0, order)
    cls, nslot, slots, coef, V = _tables(c)
    h = c.params["radius"]
    x0 = c.xyz.mean(axis=0)

    def field(p):
        s = (p - x0) / h
        f = 1.0 + 0.3 * s[..., 0] - 0.2 * s[..., 1]
        if c.dim == 3:
            f = f + 0.25 * s[..., 2]
        if order >= 2:
            f = f + 0.1 * s[..., 0] ** 2 - 0.05 * s[..., 0] * s[..., 1] + 0.07 * s[..., 1] ** 2
            if c.dim == 3:
                f = f + 0.04 * s[..., 2] ** 2 + 0.06 * s[..., 0] * s[..., 2] \
                    - 0.03 * s[..., 1] * s[..., 2]
        return f

    v = _velocities(c, V)
    worst, checked = 0.0, 0
    for i in np.nonzero(c.boundary == 0)[0]:
        n = nslot[i]
        cc = coef[cls[i], 1:n, :]                       # the neighbours' coefficients
        fs = field(c.xyz[slots[i, 1:n]])               # the field at the neighbours
        got = fs @ cc                                  # per velocity node
        foot = c.xyz[i][None, :] - (v - c.meshv[i][None, :]) * c.dt
        want = field(foot)
        worst = max(worst, float(np.abs(got - want).max() / np.abs(want).max()))
        checked += 1
    assert checked > 0
    assert worst < 1e-9, worst
