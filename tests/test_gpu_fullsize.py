"""The headline configuration at full size against the reference itself.

cavity3d, Nx = 40 (64 000 particles), Nv = 10 (1 000 velocities), quadratic
MLS, the case's default dt, started from rest.  The fixture
``step_c3d_n40_v10_q_s1_s10_s50.npz`` holds the reference CPU build's own state
after steps 1, 10 and 50 (Solver/Solver.cpp:632-705 with mlsOrder = 2, written by
``tests/golden/make_golden_c3d40.py``): every particle's moments and row sums,
256 seeded full rows, and every step's transport-flag and moodCheck counts.

FP64 mode is held to the FP64 contract with margin: 1e-10 relative on every
moment field and sampled row, and the same MOOD decisions at every step.
Velocity components are measured against the largest flow speed of the
field (a component that is rounding noise at step 1, such as uy of a gas at
rest under a lid moving in x, has no scale of its own).
FP32 mode (FP32 f and reconstruction, FP64 sums) is held to its stated
error against the same fixture: 5e-5 relative on rho and T and 2e-4 on the
sampled rows.  Its flow velocities differ from the reference's by up to
about 0.04 m/s (4 % of the 1 m/s lid speed) at step 10, next to the lid, and
0.015 m/s at step 50; the bounds are 0.06 and 0.03 m/s.  That difference is the MOOD screen's, not FP32's: the
FP32 screen carries a rounding floor (64 FP32 ulps of the neighbour density)
and so takes none of the 665-1324 linear redos per step that the reference
takes from step 4 on, and an FP64 run with the screen off differs from the
reference by the same 0.04 m/s.  With the screen off in both, FP32 tracks
FP64 to 1e-4 m/s (test_fp32_tracks_fp64_without_the_screen).
"""
import numpy as np
import pytest

from conftest import golden

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu

FIXTURE = "step_c3d_n40_v10_q_s1_s10_s50.npz"
CHECKPOINTS = (1, 10, 50)
DU50 = 0.03       # m/s at step 50 (measured 0.015: the redos' difference decays)


def relmax(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def field_errors(m, ref):
    """Relative max error of rho, ux, uy, uz, T; velocities against the
    largest flow speed of the reference field."""
    uscale = max(np.abs(ref[:, 1:4]).max(), 1e-300)
    return [relmax(m[:, 0], ref[:, 0])] + \
        [float(np.abs(m[:, q] - ref[:, q]).max() / uscale) for q in (1, 2, 3)] + \
        [relmax(m[:, 4], ref[:, 4])]


@pytest.fixture(scope="module")
def fx():
    return golden(FIXTURE)


def run(fx, precision):
    """Steps the device run to the last checkpoint; the state at every
    checkpoint and the per-step decision counts."""
    c = ab.Case("cavity3d", 40, 10, -1.0, 2)
    s = ab.Solver(c, precision=precision)
    rows = fx["rows"]
    out, flags = {}, []
    for step in range(1, max(CHECKPOINTS) + 1):
        s.cudaStep(1)
        cnt = s.counters()
        assert cnt["error_word"] == 0
        flags.append([cnt["transport_flags"], cnt["mood_fail"]])
        if step in CHECKPOINTS:
            g, m = s.cudaDownloadFull()
            out[step] = dict(macro=m[:, :5].copy(), gsum=g.sum(axis=1),
                             gabs=np.abs(g).sum(axis=1), g=g[rows].copy())
            del g
    s.close()
    return out, np.array(flags)


def test_fp64_matches_reference_at_full_size(gpu, fx):
    out, flags = run(fx, 64)
    # The MOOD decisions of every step: step 1 flags every interior particle,
    # steps 4-50 a few hundred to a thousand.
    np.testing.assert_array_equal(flags, fx["flags"])
    for step in CHECKPOINTS:
        o = out[step]
        err = field_errors(o["macro"], fx[f"macro_s{step}"])
        print("FP64 vs reference at step", step, "rho ux uy uz T:", err)
        assert max(err) < 1e-10, (step, err)
        assert relmax(o["gsum"], fx[f"gsum_s{step}"]) < 1e-10
        assert relmax(o["gabs"], fx[f"gabs_s{step}"]) < 1e-10
        assert relmax(o["g"], fx[f"g_s{step}"]) < 1e-10


def test_fp32_error_against_reference_at_full_size(gpu, fx):
    out, flags = run(fx, 32)
    # Step 1 flags every interior particle in both precisions.
    assert flags[0, 0] == fx["flags"][0, 0]
    assert (flags[:, 1] == 0).all()
    errs = {}
    for step in CHECKPOINTS:
        o = out[step]
        ref = fx[f"macro_s{step}"]
        errs[step] = field_errors(o["macro"], ref)
        assert errs[step][0] < 5e-5 and errs[step][4] < 5e-5, errs[step]
        # flow velocities (up to the 1 m/s lid speed): absolute, in m/s
        du = np.abs(o["macro"][:, 1:4] - ref[:, 1:4]).max()
        print(f"FP32 vs reference at step {step}: max |du| {du:.3e} m/s")
        assert du < {1: 1e-3, 10: 0.06, 50: DU50}[step], (step, du)
        assert relmax(o["g"], fx[f"g_s{step}"]) < 2e-4
    print("FP32 vs reference, relative max error of rho ux uy uz T:", errs)


def test_fp32_tracks_fp64_without_the_screen(gpu):
    """The FP32 path's own error at full size, with the MOOD screen off in
    both precisions so that both take the same scheme at every particle:
    10 steps of FP32 against FP64 on the device."""
    c = ab.Case("cavity3d", 40, 10, -1.0, 2)
    out = {}
    for prec in (32, 64):
        cfg = c.config(prec, 0, 0, 0)
        cfg.limiter = 0
        s = ab.Solver(c, config=cfg)
        s.cudaStep(10)
        assert s.counters()["error_word"] == 0
        out[prec] = s.cudaDownloadMoments()
        s.close()
    du = np.abs(out[32][:, 1:4] - out[64][:, 1:4]).max()
    print(f"FP32 vs FP64, screen off, step 10: max |du| {du:.3e} m/s, rho "
          f"{relmax(out[32][:, 0], out[64][:, 0]):.3e}, T {relmax(out[32][:, 4], out[64][:, 4]):.3e}")
    assert du < 1e-3
    assert relmax(out[32][:, 0], out[64][:, 0]) < 1e-5
    assert relmax(out[32][:, 4], out[64][:, 4]) < 1e-5
