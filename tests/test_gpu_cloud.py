"""Cloud management around a moving body (remove, merge, refill with the
all-particle tests and neighbour rebuilds on the GPU) against the compiled
reference's own CloudManagement.cpp on the same cloud: bitwise."""
import ctypes

import numpy as np
import pytest

from alebgk4paper_b200 import Case
from oracle.oracle import RefCase, ref_library

pytestmark = pytest.mark.gpu


def _need():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if ref_library() is None:
        pytest.skip("oracle/_ref is not built")


def _ref(name, Nx, Nv, steps, shift):
    r = RefCase(name, Nx, Nv)
    r.step(steps)
    L = r.L
    L.ref_shift_body.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double]
    L.ref_manage.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
    dx = abs(r.params["dx"])
    L.ref_shift_body(r.h, 0, shift[0] * dx, shift[1] * dx, shift[2] * dx)
    return r


def _state(r):
    d = r.cloud()
    d["g"] = r.g()
    d["macro"] = r.macro()
    return d


@pytest.mark.parametrize("name,Nx,Nv,shift", [
    ("cavity2d-square", 24, 6, (1.3, 0.45, 0.0)),
    ("cavity2d-circle", 24, 6, (2.7, -0.6, 0.0)),
    ("cavity3d-cube", 16, 4, (1.3, 0.45, 0.2)),
    ("cavity3d-sphere", 16, 4, (1.6, 0.3, -0.4)),
])
def test_cloud_management_equals_reference(name, Nx, Nv, shift):
    _need()
    from alebgk4paper_b200.cloud import manage_cloud
    a = _ref(name, Nx, Nv, 3, shift)
    b = _ref(name, Nx, Nv, 3, shift)
    before = _state(a)
    bodies = np.zeros((1, 32))
    a.L.ref_get_bodies(a.h, bodies.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    cnt = (ctypes.c_int * 3)()
    b.L.ref_manage(b.h, cnt)
    d = (ctypes.c_int * 6)()
    b.L.ref_dims(b.h, d)
    b.N = d[0]
    want = _state(b)
    case = Case(name, Nx=Nx, Nv=Nv)
    got, counts, _ = manage_cloud(case, before, bodies)
    assert counts == tuple(cnt), (counts, tuple(cnt))
    assert sum(counts) > 0                       # the shift made work for it
    assert got["xyz"].shape == want["xyz"].shape
    for k in ("xyz", "meshv", "wall", "boundary", "body_id", "nnb", "nbr", "g"):
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got["macro"][:, :6], want["macro"][:, :6])


def test_merge_of_close_particles_equals_reference():
    """Two interior particles pushed closer than minDist are merged at their
    mean position with the mean distribution, as mergeCloseParticles does."""
    _need()
    from alebgk4paper_b200.cloud import manage_cloud
    name, Nx, Nv = "cavity2d-square", 24, 6
    a = _ref(name, Nx, Nv, 2, (0.0, 0.0, 0.0))
    b = _ref(name, Nx, Nv, 2, (0.0, 0.0, 0.0))
    cl = a.cloud()
    dx = abs(a.params["dx"])
    # two interior lattice neighbours away from the body and the walls
    i = int(np.flatnonzero((cl["boundary"] == 0) & (cl["xyz"][:, 0] < 0.3e-6)
                           & (cl["xyz"][:, 1] < 0.3e-6))[0])
    j = int([n for n in cl["nbr"][i, :cl["nnb"][i]] if n > i and cl["boundary"][n] == 0
             and abs(cl["xyz"][n, 1] - cl["xyz"][i, 1]) < 1e-12][0])
    x, y = cl["xyz"][j, 0] - 0.3 * dx, cl["xyz"][j, 1]
    for r in (a, b):
        r.L.ref_set_position.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double]
        r.L.ref_set_position(r.h, i, x, y, 0.0)
    before = _state(a)
    bodies = np.zeros((1, 32))
    a.L.ref_get_bodies(a.h, bodies.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    cnt = (ctypes.c_int * 3)()
    b.L.ref_manage(b.h, cnt)
    d = (ctypes.c_int * 6)()
    b.L.ref_dims(b.h, d)
    b.N = d[0]
    want = _state(b)
    got, counts, _ = manage_cloud(Case(name, Nx=Nx, Nv=Nv), before, bodies)
    assert counts == tuple(cnt) and counts[1] >= 1
    for k in ("xyz", "boundary", "body_id", "nnb", "nbr", "g"):
        assert np.array_equal(got[k], want[k]), k
    # The same management in plan mode (no distribution passed): the row
    # plan applied to the input rows gives the managed distribution bitwise.
    geo = {k: v for k, v in before.items() if k != "g"}
    pl, pcounts, _ = manage_cloud(Case(name, Nx=Nx, Nv=Nv), geo, bodies, plan=True)
    assert pcounts == counts and pl["g"] is None
    pa, pb, fresh = pl["plan"]
    g0 = before["g"]
    rows = np.where((pb >= 0)[:, None], 0.5 * (g0[pa] + g0[np.maximum(pb, 0)]), g0[pa])
    if len(fresh):
        rows[pa < 0] = fresh[-1 - pa[pa < 0]]
    assert (pb >= 0).sum() == counts[1]
    np.testing.assert_array_equal(rows, got["g"])
    for k in ("xyz", "boundary", "body_id", "nnb", "nbr", "macro"):
        assert np.array_equal(pl[k], got[k]), k


@pytest.mark.parametrize("name,Nx,Nv,v", [("cavity2d-square", 24, 6, (900.0, 300.0, 0.0)),
                                          ("cavity3d-cube", 12, 4, (700.0, 0.0, 400.0))])
def test_fast_body_run_manages_the_cloud_like_the_reference(name, Nx, Nv, v):
    """A body launched fast enough to sweep the lattice within a few steps:
    fluid step, body step and cloud management every step, against the
    compiled reference's moving-body run.  The particle count follows the
    reference's removals and refills step for step, and the body history
    agrees to 1e-8 (the fluid steps differ in rounding only)."""
    _need()
    from alebgk4paper_b200 import Solver
    r = RefCase(name, Nx, Nv)
    r.L.ref_set_body_velocity.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double]
    r.L.ref_set_body_velocity(r.h, 0, *v)
    c = Case(name, Nx=Nx, Nv=Nv)
    st = c.bodies.copy()
    st[0, 3:6] = v
    c.bodies = st
    s = Solver(c, precision=64)
    changed = 0
    for k in range(8):
        r.step(1)
        s.cudaStep(1)
        st = s.body_step(st)
        c.bodies = st
        counts = s.refresh_geometry()
        changed += sum(counts)
        assert c.N == r.N, (k, c.N, r.N, counts)
        rb = np.zeros((1, 32))
        r.L.ref_get_bodies(r.h, rb.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        for sl in (slice(0, 3), slice(3, 6)):
            assert np.abs(st[0, sl] - rb[0, sl]).max() <= 1e-8 * np.abs(rb[0, sl]).max()
    assert changed > 0
    g_ours, _ = s.cudaDownloadFull()
    g_ref = r.g()
    assert np.abs(g_ours - g_ref).max() <= 1e-9 * np.abs(g_ref).max()
    s.close()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name,Nx,Nv,v", [("cavity2d-square", 24, 6, (900.0, 300.0, 0.0)),
                                          ("cavity3d-cube", 12, 4, (700.0, 0.0, 400.0))])
def test_particle_set_changes_keep_the_state_on_the_device(name, Nx, Nv, v, precision):
    """The fast-body run with its removals, merges and refills, once with the
    distribution kept on the device across every particle-set change (the
    management's row plan, ``alebgk_rows_build``) and once through the host
    (download, host management, upload): the same particle counts and
    bitwise the same body history, distribution and macros at every step."""
    _need()
    from alebgk4paper_b200 import Solver
    runs = []
    for device_state in (True, False):
        c = Case(name, Nx=Nx, Nv=Nv)
        st = c.bodies.copy()
        st[0, 3:6] = v
        c.bodies = st
        s = Solver(c, precision=precision)
        hist = []
        changed = [0, 0, 0]
        for _ in range(8):
            s.cudaStep(1)
            st = s.body_step(st)
            c.bodies = st
            counts = s.refresh_geometry(device_state=device_state)
            changed = [x + y for x, y in zip(changed, counts)]
            g, m = s.cudaDownloadFull()
            hist.append((c.N, st.copy(), g, m))
        runs.append((hist, changed))
        s.close()
    (ha, ca), (hb, cb) = runs
    print("removed, merged, added over the run:", ca)
    assert ca == cb and sum(ca) > 0, (ca, cb)
    for (na, sa, ga, ma), (nb, sb, gb, mb) in zip(ha, hb):
        assert na == nb
        np.testing.assert_array_equal(sa, sb)
        np.testing.assert_array_equal(ga, gb)
        np.testing.assert_array_equal(ma, mb)
