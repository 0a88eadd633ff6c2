"""State transfers through the C-ABI: alebgk_upload_state puts the host
rows on the device as the device conversion would (FP64: unchanged; FP32:
each value rounded to the nearest FP32, ties to even), and
alebgk_download_full / alebgk_download_moments bring them back.  An FP32
upload of at least 32 MB of rows converts on the host into a pinned ring of
about 8 MB row chunks while the copy engine moves the previous chunk;
cavity3d Nx=30 Nv=10 is 108 MB of FP32 rows, so the ring wraps several
times."""
import ctypes

import numpy as np
import pytest

import alebgk4paper_b200 as ab
from alebgk4paper_b200 import _abi

pytestmark = pytest.mark.gpu


def _state(N, gs, seed):
    rng = np.random.default_rng(seed)
    g = rng.lognormal(-20.0, 3.0, size=(N, gs))          # magnitudes 1e-13 .. 1e-5
    g[::97, 5] = 0.0
    g[1::89, 7] = -g[1::89, 7]                           # negative values
    # exact ties between two adjacent FP32 numbers round to even
    a = np.float32(1.0e-6)
    b = np.nextafter(a, np.float32(1.0))
    g[2::83, 3] = (np.float64(a) + np.float64(b)) / 2.0
    g[3::79, 4] = 1.0e-41                                # FP32 subnormal range
    return g


@pytest.mark.parametrize("precision,Nx", [(32, 30), (64, 30), (32, 12)])
def test_state_upload_rounds_each_value_once(gpu, precision, Nx):
    """Nx 30: the host-rounding ring (108 MB of FP32 rows); Nx 12: below the
    ring's 32 MB threshold, the device conversion."""
    c = ab.Case("cavity3d", Nx, 10, -1.0, 2)
    s = ab.Solver(c, precision=precision)
    g = _state(s.N, s.gstride, 11)
    m = np.array(c.macro, dtype=np.float64, copy=True)
    m[::5, 6] = 1.0
    m[1::5, 6] = 0.0
    dp = lambda x: x.ctypes.data_as(_abi.c_double_p)
    assert s.lib.alebgk_upload_state(s.ctx, dp(g), dp(m)) == 0
    g2, m2 = s.cudaDownloadFull()
    want = g.astype(np.float32).astype(np.float64) if precision == 32 else g
    np.testing.assert_array_equal(g2, want)
    np.testing.assert_array_equal(m2[:, :6], m[:, :6])
    np.testing.assert_array_equal(m2[:, 6], (m[:, 6] != 0.0).astype(np.float64))
    # a second upload of other values reuses the staging
    g3 = _state(s.N, s.gstride, 12)
    assert s.lib.alebgk_upload_state(s.ctx, dp(g3), dp(m)) == 0
    g4, _ = s.cudaDownloadFull()
    want = g3.astype(np.float32).astype(np.float64) if precision == 32 else g3
    np.testing.assert_array_equal(g4, want)
    s.close()


def test_uploading_the_context_state_again_changes_nothing(gpu):
    """Right after construction (mass scale exactly 1) a context's own state,
    downloaded and uploaded again through alebgk_upload_state, steps to the
    same bits as a context that was left alone: the upload restores the
    distribution, the macros, the MOOD flags and the mass reference (FP32)."""
    c = ab.Case("cavity3d", 12, 6, -1.0, 2)
    s1 = ab.Solver(c, precision=32)
    s2 = ab.Solver(c, precision=32)
    g, m = s2.cudaDownloadFull()
    dp = lambda x: np.ascontiguousarray(x).ctypes.data_as(_abi.c_double_p)
    assert s2.lib.alebgk_upload_state(s2.ctx, dp(g), dp(m)) == 0
    s1.cudaStep(5)
    s2.cudaStep(5)
    g1, m1 = s1.cudaDownloadFull()
    g2, m2 = s2.cudaDownloadFull()
    np.testing.assert_array_equal(g2, g1)
    np.testing.assert_array_equal(m2, m1)
    s1.close()
    s2.close()
