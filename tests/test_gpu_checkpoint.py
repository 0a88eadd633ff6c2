"""Restart files written from the device: the reference's own ckpt::restore
reads them and steps on to the same state, and a restore into a fresh
context continues the run."""
import numpy as np
import pytest

from conftest import ref_available

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_device_checkpoint_restores_in_the_reference(gpu, tmp_path):
    from oracle.oracle import RefCase
    c = ab.Case("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=64)
    s.cudaStep(2)
    path = str(tmp_path / "dev.ckpt")
    s.checkpoint_save(path, step=2, t=2 * c.dt)
    g, m = s.cudaDownloadFull()
    r = RefCase("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=True)
    ok, step, t = r.checkpoint_load(path)
    assert ok and step == 2 and t == pytest.approx(2 * c.dt, rel=1e-15)
    np.testing.assert_array_equal(r.g(), g)
    np.testing.assert_array_equal(r.macro()[:, :6], m[:, :6])
    # both continue from the restart to the same state
    r.step(1)
    s.cudaStep(1)
    g2, m2 = s.cudaDownloadFull()
    assert rel(g2, r.g()) < 1e-10
    assert rel(m2[:, 0], r.macro()[:, 0]) < 1e-10
    s.close()


@pytest.mark.parametrize("precision,tol", [(64, 1e-13), (32, 1e-6)])
def test_restore_continues_the_run(gpu, tmp_path, precision, tol):
    """20x20x20 x 1000 velocities: the FP64 image of g is 64 MB, copied in
    several chunks through the two pinned buffers."""
    c = ab.Case("cavity3d", 20, 10, -1.0, 2)
    a = ab.Solver(c, precision=precision)
    a.cudaStep(3)
    path = str(tmp_path / "run.ckpt")
    a.checkpoint_save(path, step=3, t=3 * c.dt)
    h = ab.read_checkpoint(path)
    assert h["N"] == c.N and h["gstride"] == c.gstride and h["step"] == 3
    b = ab.Solver(ab.Case("cavity3d", 20, 10, -1.0, 2), precision=precision)
    d = b.checkpoint_restore(path)
    assert d["step"] == 3
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    if precision == 64:
        np.testing.assert_array_equal(gb, ga)
    else:
        # the file holds h * scale in FP64; a restore stores it as h (FP32)
        # with scale 1, one FP32 rounding away from the running state
        assert rel(gb, ga) <= 2.0 ** -23
    np.testing.assert_array_equal(mb[:, :6], ma[:, :6])
    a.cudaStep(2)
    b.cudaStep(2)
    ga, ma = a.cudaDownloadFull()
    gb, mb = b.cudaDownloadFull()
    assert rel(gb, ga) < tol
    assert rel(mb[:, 0], ma[:, 0]) < tol
    a.close()
    b.close()
