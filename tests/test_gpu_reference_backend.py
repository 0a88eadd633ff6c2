"""The reference's own GPU path, compiled for sm_100a, computes the case that
the timed comparison runs.

``oracle/_ref/libalebgk_refcuda.so`` is the reference's set-up and its CUDA
backend Solver/CudaBackend.cu, compiled unmodified (``make -C oracle
refcuda``).  Two cudaStep calls of cavity3d (Nx 8, Nv 6, quadratic MLS) on it
are held to the reference CPU build's two steps and to this library's FP64
path, to the FP64 contract of 1e-6 relative on rho and T: the reference
backend assembles and solves each MLS system per node with a Cholesky
factorisation (Solver/CudaBackend.cu:699-869) where the CPU build uses
pivoted elimination, so the two agree to rounding, not bitwise.
"""
import numpy as np
import pytest

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_reference_cuda_backend_matches_cpu_build_and_this_library(gpu):
    from oracle.oracle import RefCase, ref_cuda_library, ref_library
    lib = ref_cuda_library()
    if lib is None or ref_library() is None:
        pytest.skip("oracle/_ref/libalebgk_refcuda.so not built")
    gpu_ref = RefCase("cavity3d", 8, 6, -1.0, 2, fixed_body=True, lib_path=lib)
    ms = gpu_ref.cuda_run(0, 2)
    assert ms > 0
    m_gpu = gpu_ref.macro()
    cpu_ref = RefCase("cavity3d", 8, 6, -1.0, 2, fixed_body=True)
    cpu_ref.step(2)
    m_cpu = cpu_ref.macro()
    s = ab.Solver(ab.Case("cavity3d", 8, 6, -1.0, 2), precision=64)
    s.cudaStep(2)
    m_ours = s.cudaDownloadMoments()
    s.close()
    for q in (0, 4):
        assert rel(m_gpu[:, q], m_cpu[:, q]) < 1e-6, q
        assert rel(m_ours[:, q], m_cpu[:, q]) < 1e-10, q
        assert rel(m_gpu[:, q], m_ours[:, q]) < 1e-6, q
