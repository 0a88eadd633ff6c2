"""The reference's own executable stepping on this library.

``oracle/_ref/alebgk_dropin`` is the reference's unmodified TestCases/main.cpp
and Solver/Solver.cpp (built with ALEBGK_WITH_CUDA, the build whose time loop
Solver/Solver.cpp:253-578 calls the CUDA backend of Solver/Solver.cpp:67-89),
with alebgk4paper_b200/shim/cuda_backend_shim.cpp in place of
Solver/CudaBackend.cu and libalebgk_b200.so on the link line
(``make -C oracle dropin``, where the reference sources are present; the
built binary travels with the tree).

The run is the reference's own: its CLI, case set-up, initial condition,
time loop and, with ALEBGK_CHECKPOINT_EVERY=2, its own checkpoint writer
(ckpt::save after cudaDownloadFull, Solver/Solver.cpp:565-572).  The restart
file it writes after two steps of cavity3d (Nx 8, Nv 6, the shipped linear
MLS) is compared with the compiled reference CPU build after the same two
steps: FP64 (ALEBGK_B200_PRECISION=64) to 1e-10 relative, FP32 to its stated
5e-5 on rho and T.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, ref_available

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "oracle", "_ref", "alebgk_dropin")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def reference_state():
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    from oracle.oracle import RefCase
    r = RefCase("cavity3d", 8, 6, -1.0, 1)
    dt = float(r.dt)
    r.step(2)
    return dt, r.g(), r.macro()


@pytest.mark.parametrize("precision,tol", [(64, 1e-10), (32, 5e-5)])
def test_reference_executable_runs_on_the_library(gpu, tmp_path, reference_state, precision,
                                                  tol):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/alebgk_dropin not built (make -C oracle dropin)")
    dt, g_ref, m_ref = reference_state
    env = dict(os.environ, ALEBGK_CHECKPOINT_EVERY="2", ALEBGK_B200_PRECISION=str(precision),
               OMP_NUM_THREADS="4")
    out = subprocess.run([DROPIN, "cavity3d", "--Nx", "8", "--Nv", "6", "--tfinal",
                          repr(2.0 * dt)], cwd=tmp_path, env=env, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "Steps=2" in out.stdout, out.stdout[-2000:]
    ck = ab.read_checkpoint(str(tmp_path / "output" / "cavity3d_Nx8_Nv6" / "restart.ckpt"))
    assert ck["step"] == 2 and ck["N"] == g_ref.shape[0]
    m = ck["macro"]
    assert rel(m[:, 0], m_ref[:, 0]) < tol
    assert rel(m[:, 4], m_ref[:, 4]) < tol
    # flow velocities against the largest flow speed of the field
    utol = tol if precision == 64 else 1e-3
    uscale = np.abs(m_ref[:, 1:4]).max()
    assert np.abs(m[:, 1:4] - m_ref[:, 1:4]).max() / uscale < utol
    if precision == 64:
        assert rel(ck["g"], g_ref) < tol
