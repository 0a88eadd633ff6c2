"""Batches of independent cavities: one graph launch per step gives each
cavity exactly the state it reaches on its own, the residuals agree with the
per-cavity ones, autotuning changes only launch shapes, and a small batch
runs to a steady residual."""
import numpy as np
import pytest

import alebgk4paper_b200 as ab
from alebgk4paper_b200.batch import BatchSolver, batched_cavity2d

pytestmark = pytest.mark.gpu

SPECS = [
    dict(name="cavity2d", Nx=12, Nv=8, lid_speed=1.0, rho0=1.0, tau=3.7142e-10, dt=2e-12),
    dict(name="cavity2d", Nx=16, Nv=10, lid_speed=5.0, rho0=3.0, tau=3.7142e-10 / 3,
         dt=3e-12),
    dict(name="cavity3d", Nx=8, Nv=6, lid_speed=2.0, rho0=1.5, tau=3.7142e-10 / 1.5,
         dt=5e-12),
]


def _alone(spec, precision, steps):
    kw = dict(spec)
    name = kw.pop("name")
    s = ab.Solver(ab.Case(name, **kw), precision=precision)
    s.cudaStep(steps)
    g, m = s.cudaDownloadFull()
    r = s.residual()
    s.close()
    return g, m, r


@pytest.mark.parametrize("precision", [32, 64])
def test_batch_graph_equals_each_cavity_alone(gpu, precision):
    b = BatchSolver(SPECS, precision=precision)
    b.step(4)
    res = b.residuals()
    for i, sp in enumerate(SPECS):
        g0, m0, r0 = _alone(sp, precision, 4)
        g1, m1 = b.solvers[i].cudaDownloadFull()
        np.testing.assert_array_equal(g1, g0)
        np.testing.assert_array_equal(m1, m0)
        assert res[i] == r0
    # the contexts stay usable on their own, in step with the batch
    b.solvers[0].cudaStep(1)
    b.solvers[1].cudaStep(1)
    b.solvers[2].cudaStep(1)
    b.step(1)
    b.close()


def test_autotune_changes_only_launch_shapes(gpu):
    sp = dict(SPECS[1])
    name = sp.pop("name")
    a = ab.Solver(ab.Case(name, **sp), precision=32)
    t = ab.Solver(ab.Case(name, **sp), precision=32)
    ms = t.autotune(2)
    assert ms > 0
    tt, pw = t.get_launch()
    assert tt in (0, 64, 128, 256) and pw in (0, 1, 2, 4)
    a.cudaStep(5)
    t.cudaStep(5)
    np.testing.assert_array_equal(t.cudaDownloadFull()[0], a.cudaDownloadFull()[0])
    a.close()
    t.close()


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("name", ["cavity2d", "cavity3d"])
def test_fused_transport_equals_separate_kernels(gpu, precision, name):
    """Transport inside the particle kernel (transport threads 0) gives the
    bitwise state of the separate transport kernel, MOOD redos included."""
    sp = dict(SPECS[1] if name == "cavity2d" else SPECS[2])
    sp.pop("name")
    out = []
    for tt in (0, 128):
        s = ab.Solver(ab.Case(name, **sp), precision=precision)
        s.set_launch(tt, 0)
        s.cudaStep(6)
        out.append(s.cudaDownloadFull())
        s.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_small_batch_runs_to_steady(gpu):
    """Four seeded cavities at the workload's smallest grids (Nx=24, Nv=16)
    reach the steady residual 1e-6.  The residual floor is the per-step mass
    drift of the discrete collision, about 1e-8 (the reference's own CPU
    path drifts the same way), far below it."""
    specs = batched_cavity2d(4, seed=3, Nx_choices=(24,), Nv_choices=(16,))
    b = BatchSolver(specs, precision=32, autotune=True, tune_steps=2)
    done = b.run_to_steady(tol=1e-6, check_every=100, max_steps=10000)
    assert (done > 0).all()
    assert (b.residuals() < 1e-6).all()
    b.close()


def test_uneven_batch_with_smallest_rows_last(gpu):
    """Cavities with different velocity grids in one batch, the smallest rows
    uploaded last: every context's kernels must stay launchable (the shared
    memory cap of a kernel is shared by all contexts of the process)."""
    specs = [dict(name="cavity2d", Nx=24, Nv=nv, lid_speed=2.0, rho0=1.0, tau=3.7142e-10,
                  dt=1.25 * (1e-6 / 23) / 1303.0, mls_order=2) for nv in (24, 20, 16)]
    b = BatchSolver(specs, precision=32)
    b.step(4)
    b.sync()
    alone = [BatchSolver([sp], precision=32) for sp in specs]
    for a in alone:
        a.step(4)
        a.sync()
    for s, a in zip(b.solvers, alone):
        np.testing.assert_array_equal(s.cudaDownloadFull()[0], a.solvers[0].cudaDownloadFull()[0])
        a.close()
    b.close()


@pytest.mark.parametrize("precision", [32, 64])
def test_stage_launches_equal_each_cavity_alone(gpu, precision):
    """Uneven 2-D cavities of the batched workload advanced by one launch per
    stage over the whole batch: every cavity's distribution, macros and
    residual are bitwise those of its own step, and the same as the graph of
    per-cavity branches."""
    specs = batched_cavity2d(5, seed=7)
    b = BatchSolver(specs, precision=precision)
    br = BatchSolver(specs, precision=precision, launch="branches")
    b.step(6)
    br.step(6)
    assert b.staged and not br.staged
    res, res_br = b.residuals(), br.residuals()
    for i, sp in enumerate(specs):
        g0, m0, r0 = _alone(sp, precision, 6)
        g1, m1 = b.solvers[i].cudaDownloadFull()
        g2, m2 = br.solvers[i].cudaDownloadFull()
        np.testing.assert_array_equal(g1, g0)
        np.testing.assert_array_equal(m1, m0)
        np.testing.assert_array_equal(g2, g0)
        assert res[i] == r0 and res_br[i] == r0
    b.close()
    br.close()


def test_mixed_batch_falls_back_to_branches(gpu):
    """2-D and 3-D cavities (one and two Chu layers) cannot share stage
    launches; the batch uses per-cavity branches."""
    b = BatchSolver(SPECS, precision=32)
    b.step(1)
    assert not b.staged
    b.close()


def test_batch_autotune_keeps_states_exact(gpu):
    """The batch autotuner's timed steps (stage groups 1, 2, 4, the
    persistent launch and per-cavity branches) are real steps: afterwards
    every cavity holds exactly the state of as many steps on its own."""
    specs = batched_cavity2d(5, seed=11)
    b = BatchSolver(specs, precision=32)
    ms = b.autotune(2)
    assert ms > 0
    assert b.steps == 5 * (2 + 2)
    b.step(1)
    for i, sp in enumerate(specs):
        g0, m0, _ = _alone(sp, 32, b.steps)
        g1, m1 = b.solvers[i].cudaDownloadFull()
        np.testing.assert_array_equal(g1, g0)
        np.testing.assert_array_equal(m1, m0)
    b.close()


@pytest.mark.parametrize("launch", ["stages", "branches", "persistent"])
def test_batch_recaptures_after_a_context_is_uploaded_again(gpu, launch):
    """A context uploaded again between batch steps has new buffers: the
    batch notices (upload epoch) and rebuilds its graphs, so the cavity
    restarts from its upload and the others carry on, each exactly as alone."""
    specs = batched_cavity2d(3, seed=5)
    b = BatchSolver(specs, precision=32, launch=launch)
    b.step(2)
    b.sync()
    b.solvers[0].cudaUploadCloud(b.cases[0])
    b.step(2)
    g0, m0, _ = _alone(specs[0], 32, 2)
    np.testing.assert_array_equal(b.solvers[0].cudaDownloadFull()[0], g0)
    for i in (1, 2):
        gi, mi, _ = _alone(specs[i], 32, 4)
        np.testing.assert_array_equal(b.solvers[i].cudaDownloadFull()[0], gi)
    b.close()


@pytest.mark.parametrize("precision", [32, 64])
def test_persistent_launch_equals_each_cavity_alone(gpu, precision):
    """The whole step of the batch in one persistent cooperative launch
    (every stage's blocks over the resident grid, a grid barrier between
    stages): every cavity's distribution, macros and residual are bitwise
    those of its own step."""
    specs = batched_cavity2d(6, seed=13)
    b = BatchSolver(specs, precision=precision, launch="persistent")
    b.step(5)
    assert b.staged == 1 and b.launch == "persistent"
    res = b.residuals()
    for i, sp in enumerate(specs):
        g0, m0, r0 = _alone(sp, precision, 5)
        g1, m1 = b.solvers[i].cudaDownloadFull()
        np.testing.assert_array_equal(g1, g0)
        np.testing.assert_array_equal(m1, m0)
        assert res[i] == r0
        assert b.solvers[i].counters()["error_word"] == 0
    b.close()


def test_persistent_request_falls_back_to_branches(gpu):
    """Cavities that cannot share stage launches (2-D and 3-D, the lattice
    march) run as per-cavity branches when the persistent launch is asked
    for, each exactly as alone."""
    b = BatchSolver(SPECS, precision=32, launch="persistent")
    b.step(2)
    assert b.staged == 0
    for i, sp in enumerate(SPECS):
        g0, _, _ = _alone(sp, 32, 2)
        np.testing.assert_array_equal(b.solvers[i].cudaDownloadFull()[0], g0)
    b.close()


def test_persistent_barrier_gives_up_with_an_error(gpu):
    """A grid barrier allowed no polls gives up at once: the launch ends,
    bit 8 of the first cavity's error word is set and the host sees
    ALEBGK_EDEVICE -- no wait without end on the device."""
    specs = batched_cavity2d(3, seed=3)
    b = BatchSolver(specs, precision=32, launch="persistent")
    b.set_spin_limit(0)
    b.step(1)
    b.sync()
    assert b.solvers[0].counters()["error_word"] & 8
    with pytest.raises(ab.AlebgkError):
        b.solvers[0].sync()
    b.close()
