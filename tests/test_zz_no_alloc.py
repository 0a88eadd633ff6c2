"""alebgk_body_loads_noalloc -- body loads from a fixed device scratch -- gives
the loads of the allocating alebgk_body_loads (RigidBody/BodyDynamics.cpp:17-97)
to rounding, call after call.  Collected last on purpose: it must pass alone
and after every other test of the session."""
import ctypes

import numpy as np
import pytest

import alebgk4paper_b200 as ab
from alebgk4paper_b200 import _abi

pytestmark = pytest.mark.gpu

# Per-block then over-block sums instead of one serial sum: FP64 rounding only.
RTOL = 1e-10


def _noalloc(s, centres, areas):
    nb = len(areas)
    c = np.ascontiguousarray(centres, np.float64).reshape(nb, 3)
    a = np.ascontiguousarray(areas, np.float64)
    out = np.zeros((nb, 6))
    rc = s.lib.alebgk_body_loads_noalloc(s.ctx, nb, c.ctypes.data_as(_abi.c_double_p),
                                         a.ctypes.data_as(_abi.c_double_p),
                                         out.ctypes.data_as(_abi.c_double_p))
    assert rc == _abi.OK
    return out


@pytest.mark.parametrize("name,nx,nv,precision", [
    ("cavity3d-cube", 12, 4, 64),
    ("cavity3d-cube", 12, 4, 32),
    ("cavity2d-square", 24, 8, 64),
    ("cavity2d-circle", 24, 8, 32),
])
def test_noalloc_matches_allocating_loads(gpu, name, nx, nv, precision):
    c = ab.Case(name, nx, nv, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=precision)
    s.cudaStep(2)
    centres, areas = c.bodies[:, 0:3], c.bodies[:, 31]
    want = s.body_loads(centres, areas)
    first = _noalloc(s, centres, areas)
    second = _noalloc(s, centres, areas)
    scale = np.abs(want).max()
    assert scale > 0
    assert np.abs(first - want).max() <= RTOL * scale
    assert np.abs(second - want).max() <= RTOL * scale
    assert np.array_equal(first, second)
    # the state moves on; the scratch holds nothing over from the last call
    s.cudaStep(1)
    want3 = s.body_loads(centres, areas)
    got3 = s.body_loads_noalloc(centres, areas)
    assert np.abs(got3 - want3).max() <= RTOL * np.abs(want3).max()
    s.close()


def test_noalloc_rejects_too_many_bodies(gpu):
    c = ab.Case("cavity2d-square", 16, 6, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=64)
    nb = _abi.NOALLOC_MAX_BODIES + 1
    cen = np.zeros((nb, 3))
    area = np.ones(nb)
    out = np.zeros((nb, 6))
    rc = s.lib.alebgk_body_loads_noalloc(s.ctx, nb, cen.ctypes.data_as(_abi.c_double_p),
                                         area.ctypes.data_as(_abi.c_double_p),
                                         out.ctypes.data_as(_abi.c_double_p))
    assert rc == _abi.EINVAL
    buf = ctypes.create_string_buffer(256)
    s.lib.alebgk_last_error(s.ctx, buf, 256)
    assert str(_abi.NOALLOC_MAX_BODIES) in buf.value.decode()
    assert s.lib.alebgk_body_loads_noalloc(s.ctx, 0, cen.ctypes.data_as(_abi.c_double_p),
                                           area.ctypes.data_as(_abi.c_double_p),
                                           out.ctypes.data_as(_abi.c_double_p)) == _abi.EINVAL
    # a rejected call leaves the context usable
    got = s.body_loads_noalloc(c.bodies[:, 0:3], c.bodies[:, 31])
    want = s.body_loads(c.bodies[:, 0:3], c.bodies[:, 31])
    assert np.abs(got - want).max() <= RTOL * np.abs(want).max()
    s.close()
