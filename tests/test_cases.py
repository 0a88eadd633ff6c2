"""The host case set-up reproduces the reference's clouds
(TestCases/TestCases.cpp:113-294, Initialization/*.cpp) against fixtures
generated by the reference itself."""
import numpy as np
import pytest

from conftest import golden, ref_available
from tests.golden.make_golden import SETUPS, nbr_hash

import alebgk4paper_b200 as ab


@pytest.mark.parametrize("case,Nx,Nv,order,fixed", SETUPS)
def test_setup_matches_reference_fixture(case, Nx, Nv, order, fixed):
    fx = golden(f"setup_{case}_n{Nx}_v{Nv}.npz")
    c = ab.Case(case, Nx, Nv, -1.0, order, fixed_body=fixed)
    assert c.N == len(fx["boundary"])
    np.testing.assert_allclose(c.xyz, fx["xyz"], rtol=0, atol=1e-20)
    np.testing.assert_allclose(c.wall, fx["wall"], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(c.boundary, fx["boundary"])
    np.testing.assert_array_equal(c.body_id, fx["body_id"])
    np.testing.assert_array_equal(c.nnb, fx["nnb"])
    # same neighbour lists in the same order
    np.testing.assert_array_equal(nbr_hash(c.nbr, c.nnb), fx["nbr_hash"])
    np.testing.assert_allclose(c.g[:4], fx["g0"], rtol=1e-14, atol=0)
    p = fx["params"]
    for k, v in zip(("dt", "tau", "R", "dx", "radius", "dv", "vmin", "rho0", "Tw"), p):
        assert c.params[k] == pytest.approx(v, rel=1e-15), k


def test_case_defaults_and_overrides():
    c = ab.Case("cavity3d", 6, 4)
    assert (c.dim, c.Nv, c.N, c.gstride) == (3, 4, 216, 64)
    assert c.params["tau"] == 3.7142e-10 and c.params["R"] == 208.0
    # foot-point clamp of Solver/Solver.cpp:183-199: dt far above CFL 1.5
    c2 = ab.Case("cavity2d", 10, 8, dt=1e-9)
    vmax = 1303.0
    assert c2.dt == pytest.approx(0.75 * c2.params["dx"] / vmax)
    c3 = ab.Case("cavity2d", 10, 8, dt=1e-12)
    assert c3.dt == 1e-12


def test_lid_and_wall_state():
    c = ab.Case("cavity3d", 6, 4)
    top = np.isclose(c.xyz[:, 2], 1e-6) & (c.boundary == 1)
    face = top & (c.xyz[:, 0] > 0) & (c.xyz[:, 0] < 1e-6) & (c.xyz[:, 1] > 0) & (c.xyz[:, 1] < 1e-6)
    assert np.all(c.wall[face, 3] == 1.0)                 # uniform lid on z = L
    assert np.allclose(c.wall[face, :3], [0, 0, -1])
    corner = np.where((c.xyz[:, 0] == 0) & (c.xyz[:, 1] == 0) & top)[0][0]
    assert np.allclose(np.linalg.norm(c.wall[corner, :3]), 1.0)
    assert c.wall[corner, 3] == pytest.approx(1.0 / 3.0)  # averaged over 3 faces
    b = ab.Case("cavity2d-square", 24, 8)
    lid = (b.boundary == 1) & (b.body_id < 0) & np.isclose(b.xyz[:, 1], 1e-6)
    s = b.xyz[lid, 0] / 1e-6
    np.testing.assert_allclose(b.wall[lid, 3], 10 * (2 * s) ** 2 * (2 - 2 * s) ** 2)


def test_body_embedding_counts():
    c = ab.Case("cavity3d-cube", 12, 4)
    assert (c.body_id >= 0).sum() == 96           # 4x4 points per face
    assert c.nbodies == 1
    m = c.bodies[0]
    L = 1.5e-7
    assert m[19] == pytest.approx(4.4 * 10 * L ** 3)   # mass
    assert m[20] == pytest.approx(m[19] * L * L / 6)   # isotropic inertia
    assert m[31] == pytest.approx(6 * L * L / 96)      # area per surface point


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case,Nx,Nv", [("cavity3d", 14, 4), ("cavity3d-cube", 20, 4),
                                         ("cavity2d-circle", 30, 8)])
def test_setup_matches_compiled_reference(case, Nx, Nv):
    from oracle.oracle import RefCase
    r = RefCase(case, Nx, Nv, -1.0, 2, fixed_body=True)
    cl = r.cloud()
    c = ab.Case(case, Nx, Nv, -1.0, 2, fixed_body=True)
    assert c.N == r.N
    np.testing.assert_allclose(c.xyz, cl["xyz"], rtol=0, atol=1e-20)
    np.testing.assert_array_equal(c.nnb, cl["nnb"])
    np.testing.assert_array_equal(c.nbr, cl["nbr"])
    np.testing.assert_allclose(c.g, r.g(), rtol=1e-14, atol=0)


def test_lattice_case_matches_host_parameters_and_bodies():
    """The device set-up's case parameters are the host set-up's, and so are
    the bodies it embeds (state, kind, rotation flag, size); the particle
    count of a case with bodies needs the device (tests/test_gpu_setup.py)."""
    import ctypes
    from alebgk4paper_b200 import Case, LatticeCase, _abi
    for name, kw in (("cavity2d", dict(Nx=24, Nv=16, lid_speed=3.0, rho0=2.0, tau=1.8e-10)),
                     ("cavity3d", dict(Nx=13, Nv=8))):
        lc, c = LatticeCase(name, **kw), Case(name, **kw)
        assert lc.params == c.params and lc.N == c.N and lc.gstride == c.gstride
        assert lc.nbodies == 0
    lib = _abi.load()
    for name, fixed, scale in (("cavity2d-square", 0, 1.0), ("cavity2d-circle", 1, 1.0),
                               ("cavity3d-sphere", 0, 0.8), ("cavity3d-cube", 1, 1.0)):
        c = Case(name, 12, 4, -1.0, 2, fixed_body=bool(fixed), body_scale=scale)
        n = ctypes.c_int()
        st, kind = np.zeros(32), np.zeros(1, np.int32)
        rot, size = np.zeros(1, np.int32), np.zeros(1)
        assert lib.alebgk_lattice_bodies(name.encode(), 12, 4, -1.0, 2, fixed, scale,
                                         ctypes.byref(n), st.ctypes.data_as(
                                             ctypes.POINTER(ctypes.c_double)),
                                         kind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                         rot.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                         size.ctypes.data_as(
                                             ctypes.POINTER(ctypes.c_double))) == 0
        assert n.value == c.nbodies == 1
        np.testing.assert_array_equal(st, c.bodies[0])
        assert (kind[0], rot[0], size[0]) == (c.body_kind[0], c.body_rotates[0],
                                              c.body_size[0])
