"""The reference's own GPU path, compiled for sm_100a, runs the case that the
timed comparison uses.

``oracle/_ref/libalebgk_refcuda.so`` is the reference's set-up and its CUDA
backend Solver/CudaBackend.cu, compiled unmodified (``make -C oracle
refcuda``).  Its MOOD screen differs from the reference's own CPU build: the
CPU step re-transports a flagged particle with linear MLS
(Solver/Solver.cpp:641-646), the CUDA backend rescales the transported row
back into its neighbours' density range (kNAD3D, Solver/CudaBackend.cu:
909-955).  The rescale changes density only, so after the first step --
where the screen flags every interior particle of the rest state -- the two
builds agree on temperature and flow velocity and differ in density.  This
library follows the CPU build (tests/test_gpu_parity.py); this test pins
what the timed reference GPU path computes: one cudaStep of cavity3d (Nx 8,
Nv 6, quadratic MLS) against the CPU build's step, temperature to 1e-10
relative and velocity to 1e-10 of the flow speed, with the density
difference printed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reference_cuda_backend_runs_the_same_case(gpu):
    from oracle.oracle import RefCase, ref_cuda_library, ref_library
    lib = ref_cuda_library()
    if lib is None or ref_library() is None:
        pytest.skip("oracle/_ref/libalebgk_refcuda.so not built")
    gpu_ref = RefCase("cavity3d", 8, 6, -1.0, 2, fixed_body=True, lib_path=lib)
    ms = gpu_ref.cuda_run(0, 1)
    assert ms > 0
    m_gpu = gpu_ref.macro()
    cpu_ref = RefCase("cavity3d", 8, 6, -1.0, 2, fixed_body=True)
    cpu_ref.step(1)
    m_cpu = cpu_ref.macro()
    dT = np.abs(m_gpu[:, 4] - m_cpu[:, 4]).max() / np.abs(m_cpu[:, 4]).max()
    du = np.abs(m_gpu[:, 1:4] - m_cpu[:, 1:4]).max() / np.abs(m_cpu[:, 1:4]).max()
    drho = np.abs(m_gpu[:, 0] - m_cpu[:, 0]).max() / np.abs(m_cpu[:, 0]).max()
    print(f"reference CUDA backend vs CPU build after one step: T {dT:.2e}, u {du:.2e}, "
          f"rho {drho:.2e} (the NAD clamp against the linear redo)")
    assert dT < 1e-10
    assert du < 1e-10
