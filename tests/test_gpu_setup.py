"""Lattice set-up on the device (``alebgk_upload_lattice``): every array the
GPU builds equals the host set-up bitwise, and a solver set up on the device
steps to exactly the state of one set up on the host."""
import numpy as np
import pytest

from alebgk4paper_b200 import Case, LatticeCase, Solver

pytestmark = pytest.mark.gpu

CASES = [
    ("cavity2d", dict(Nx=12, Nv=8)),
    ("cavity2d", dict(Nx=24, Nv=16, lid_speed=3.0, rho0=2.0, tau=1.8e-10, dt=3.0e-11)),
    ("cavity2d", dict(Nx=48, Nv=20, lid_speed=7.5, rho0=0.6, tau=6e-10, dt=2.0e-11)),
    ("cavity3d", dict(Nx=9, Nv=6)),
    ("cavity3d", dict(Nx=13, Nv=8, lid_speed=2.0)),
    ("cavity3d", dict(Nx=40, Nv=10)),
]


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("name,kw", CASES)
def test_device_lattice_equals_host_setup(name, kw):
    _need_gpu()
    host = Case(name, **kw)
    dev = LatticeCase(name, **kw).build_on_device()
    assert np.array_equal(dev["xyz"], host.xyz)
    assert np.array_equal(dev["wall"], host.wall)
    assert np.array_equal(dev["boundary"], host.boundary)
    assert np.array_equal(dev["nnb"], host.nnb)
    assert np.array_equal(dev["nbr"], host.nbr)


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name,kw", [CASES[1], CASES[4]])
def test_device_setup_steps_like_host_setup(name, kw, precision):
    _need_gpu()
    a = Solver(Case(name, **kw), precision=precision)
    b = Solver(LatticeCase(name, **kw), precision=precision)
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    assert np.array_equal(ga, gb) and np.array_equal(ma, mb)
    a.cudaStep(5)
    b.cudaStep(5)
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    assert np.array_equal(ga, gb) and np.array_equal(ma, mb)
    assert a.counters() == b.counters()
    a.cudaFreeCloud()
    b.cudaFreeCloud()


BODY_CASES = [("cavity2d-square", dict(Nx=24, Nv=8)), ("cavity2d-circle", dict(Nx=20, Nv=8)),
              ("cavity3d-sphere", dict(Nx=12, Nv=4)), ("cavity3d-cube", dict(Nx=12, Nv=4)),
              ("cavity3d-cube", dict(Nx=40, Nv=4, body_scale=1.3)),
              ("cavity2d-circle", dict(Nx=60, Nv=8, fixed_body=True))]


@pytest.mark.parametrize("name,kw", BODY_CASES)
def test_device_body_embedding_equals_host_setup(name, kw):
    """The bodies embedded on the device (BodyEmbedding.cpp:18-104): the
    same particles in the same order -- lattice particles inside a body or
    within 0.4 dx of its surface dropped, the surface particles appended --
    with the same wall state, body ids and neighbour lists as the host."""
    _need_gpu()
    host = Case(name, **kw)
    lc = LatticeCase(name, **kw)
    assert lc.N == host.N and lc.nbodies == host.nbodies == 1
    np.testing.assert_array_equal(lc.bodies, host.bodies)
    dev = lc.build_on_device()
    for k in ("xyz", "wall", "boundary", "body_id", "nnb", "nbr"):
        assert np.array_equal(dev[k], getattr(host, k)), k


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name,kw", [BODY_CASES[0], BODY_CASES[3]])
def test_device_body_setup_steps_like_host_setup(name, kw, precision):
    """A body case set up on the device steps bitwise like the host-built
    one, the body loads included."""
    _need_gpu()
    a = Solver(Case(name, **kw), precision=precision)
    b = Solver(LatticeCase(name, **kw), precision=precision)
    a.cudaStep(3)
    b.cudaStep(3)
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    assert np.array_equal(ga, gb) and np.array_equal(ma, mb)
    c = a.case
    centres = c.bodies[:, 0:3].copy()
    areas = c.bodies[:, 31].copy()
    assert np.array_equal(a.body_loads(centres, areas), b.body_loads(centres, areas))
    a.cudaFreeCloud()
    b.cudaFreeCloud()


def test_moving_body_run_from_device_setup(gpu):
    """A free cube set up on the device, stepped with its body step and
    cloud management, follows the host-built run bitwise."""
    runs = []
    for case in (Case("cavity3d-cube", 12, 4, -1.0, 2), LatticeCase("cavity3d-cube", 12, 4, -1.0, 2)):
        s = Solver(case, precision=64)
        st = case.bodies.copy()
        for _ in range(6):
            s.cudaStep(1)
            st = s.body_step(st)
            case.bodies = st
            s.refresh_geometry()
        runs.append((st.copy(), s.cudaDownloadFull()[0]))
        s.close()
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_batch_with_device_setup_matches_host_setup():
    _need_gpu()
    from alebgk4paper_b200.batch import BatchSolver, batched_cavity2d
    specs = batched_cavity2d(6, seed=5)
    a = BatchSolver(specs, setup="host")
    b = BatchSolver(specs, setup="device")
    a.step(10)
    b.step(10)
    for sa, sb in zip(a.solvers, b.solvers):
        assert np.array_equal(sa.cudaDownloadFull()[0], sb.cudaDownloadFull()[0])
    assert np.array_equal(a.residuals(), b.residuals())
    a.close()
    b.close()


@pytest.mark.parametrize("name,kw", [("cavity2d-square", dict(Nx=24, Nv=6)),
                                     ("cavity2d-circle", dict(Nx=24, Nv=6)),
                                     ("cavity3d-cube", dict(Nx=16, Nv=4)),
                                     ("cavity3d-sphere", dict(Nx=16, Nv=4)),
                                     ("cavity3d", dict(Nx=12, Nv=4))])
def test_device_neighbour_rebuild_equals_host_search(name, kw):
    """Neighbour lists of arbitrary clouds (body surface particles among the
    lattice) built on the device equal the host search bitwise."""
    _need_gpu()
    case = Case(name, **kw)
    s = Solver(case, precision=64)
    nnb, nbr = s.rebuild_neighbours()
    assert np.array_equal(nnb, case.nnb)
    assert np.array_equal(nbr, case.nbr)
    s.cudaFreeCloud()


@pytest.mark.parametrize("name,kw,precision", [
    ("cavity2d", dict(Nx=24, Nv=16), 32),
    ("cavity2d", dict(Nx=24, Nv=16), 64),
    ("cavity3d", dict(Nx=12, Nv=6), 64),
    ("cavity2d-square", dict(Nx=24, Nv=8), 32),
    ("cavity2d-circle", dict(Nx=24, Nv=8), 64),
    ("cavity3d-cube", dict(Nx=16, Nv=6), 32),
    ("cavity3d-sphere", dict(Nx=16, Nv=6), 64),
])
def test_device_mls_tables_equal_host_tables(name, kw, precision):
    """The MLS coefficient tables solved on the device (one thread per class
    and velocity node) equal the host builder's bitwise: a solver set up with
    either steps to the same state, with the same degenerate-stencil count."""
    _need_gpu()
    from alebgk4paper_b200 import _abi
    lib = _abi.load()
    case = Case(name, **kw)
    try:
        lib.alebgk_set_coeff_builder(1)
        a = Solver(case, precision=precision)
        lib.alebgk_set_coeff_builder(0)
        b = Solver(case, precision=precision)
    finally:
        lib.alebgk_set_coeff_builder(0)
    assert a.counters()["mls_degenerate"] == b.counters()["mls_degenerate"]
    a.cudaStep(5)
    b.cudaStep(5)
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    assert np.array_equal(ga, gb) and np.array_equal(ma, mb)
    a.cudaFreeCloud()
    b.cudaFreeCloud()


def test_bad_neighbour_lists_are_refused_at_the_first_bad_particle(gpu):
    """The upload and the in-place geometry refresh check every neighbour
    list (counts within 0..ALEBGK_MAX_NEIGH, indices of other particles) and
    name the first particle that fails."""
    import ctypes
    import alebgk4paper_b200 as ab
    c = ab.Case("cavity3d", 8, 4, -1.0, 2)
    good_nbr, good_nnb = c.nbr.copy(), c.nnb.copy()
    c.nbr[40, 2] = c.N                 # index past the cloud
    c.nbr[17, 0] = 17                  # itself
    with pytest.raises(ab.AlebgkError, match="neighbour index out of range at particle 17"):
        ab.Solver(c, precision=64)
    c.nbr[:], c.nnb[:] = good_nbr, good_nnb
    c.nnb[9] = -1
    with pytest.raises(ab.AlebgkError, match="neighbour count out of range at particle 9"):
        ab.Solver(c, precision=64)
    # the in-place refresh of an uploaded context (FP64: the general path)
    c.nbr[:], c.nnb[:] = good_nbr, good_nnb
    s = ab.Solver(c, precision=64)
    c.nbr[33, 1] = -5
    cl = c.cloud()
    rc = s.lib.alebgk_upload_geometry(s.ctx, ctypes.byref(cl), c.dt)
    assert rc != 0
    buf = ctypes.create_string_buffer(512)
    s.lib.alebgk_last_error(s.ctx, buf, 512)
    assert "neighbour index out of range at particle 33" in buf.value.decode()
    c.nbr[:] = good_nbr
    s.close()
