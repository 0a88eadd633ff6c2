"""Slab mode on the device: a cavity split into slabs (one context each,
global sums combined in slab order, ghost rows refreshed after every step)
steps to the state of the unsplit cavity, up to the summation order of the
global mass sums."""
import numpy as np
import pytest

from alebgk4paper_b200 import Case, Solver
from alebgk4paper_b200.slab import SlabGroup

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("name,kw,n,precision,tol", [
    ("cavity2d", dict(Nx=32, Nv=16, lid_speed=5.0), 2, 64, 1e-12),
    ("cavity2d", dict(Nx=33, Nv=12, lid_speed=8.0), 3, 64, 1e-12),
    ("cavity3d", dict(Nx=24, Nv=8, lid_speed=10.0), 2, 64, 1e-12),
    ("cavity3d", dict(Nx=24, Nv=8, lid_speed=10.0), 2, 32, 2e-6),
])
def test_slabs_step_like_the_whole_cavity(name, kw, n, precision, tol):
    _need_gpu()
    case = Case(name, **kw)
    whole = Solver(case, precision=precision)
    group = SlabGroup(case, n, precision=precision)
    assert abs(group.total_mass() - whole.cudaTotalMass()) <= 1e-13 * whole.cudaTotalMass()
    for _ in range(3):
        whole.cudaStep(4)
        group.step(4)
        gw, mw = whole.cudaDownloadFull()
        gs, ms = group.download_full()
        assert np.abs(gs - gw).max() <= tol * np.abs(gw).max()
        assert np.abs(ms[:, :6] - mw[:, :6]).max(0).max() <= \
            tol * np.abs(mw[:, :6]).max()
        m_whole, m_slab = whole.cudaTotalMass(), group.total_mass()
        # The step's mass change is the collision's: the discrete
        # Maxwellian's mass differs from rho by a function of (u, T) (its
        # discretisation error), weighted by dt/tau.  In FP64 the two runs
        # agree up to summation order; in FP32 their macros differ by the
        # FP32 transport's rounding (~1e-6 relative, of random sign), so the
        # masses part by ~1e-11 over the 12 steps.
        mtol = 1e-12 if precision == 64 else 1e-9
        assert abs(m_slab - m_whole) <= mtol * m_whole
    group.close()
    whole.cudaFreeCloud()
