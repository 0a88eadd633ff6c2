"""GPU parity of the B200 step, through the C-ABI, against the C oracle (same
inputs, same step count) and against the reference's own golden fixtures.

Tolerances: FP64 mode must agree with the FP64 oracle to 1e-10 relative on
every field (the contract is 1e-6); FP32 mode (FP32 f storage and FP32 MLS
reconstruction, FP64 sums) is held to 5e-5 relative on rho and T and 1e-4 on
the distribution after a few steps.  FP32 rounding of f (6e-8) is amplified
by the MLS fit (sum |c_s| of 2-5) each step; the quadratic cavity2d run at
CFL 0.002 amplifies most, as the reference's own instability at small CFL
(TestCases/TestCases.cpp:179-184) suggests.
"""
import numpy as np
import pytest

from conftest import golden
from tests.golden.make_golden import LONG_STEPS, STEPS

import alebgk4paper_b200 as ab
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


CASES = [
    ("cavity2d", 20, 16, 2, 10),      # the CPU-runnable config's grid
    ("cavity2d", 12, 8, 1, 6),        # linear MLS
    ("cavity3d", 8, 6, 2, 4),         # step 1 flags every interior particle
    ("cavity3d", 9, 5, 2, 3),         # odd Nv: a v = 0 node on every axis
    ("cavity3d", 12, 10, 2, 4),       # the bench's velocity grid
    ("cavity3d", 8, 6, 1, 3),
    ("cavity2d-square", 24, 8, 2, 4),
    ("cavity2d-circle", 20, 8, 2, 3),
    ("cavity3d-cube", 12, 4, 2, 2),   # irregular cloud round a body
    ("cavity3d-sphere", 12, 4, 2, 2),
]


@pytest.mark.parametrize("case,Nx,Nv,order,steps", CASES)
def test_fp64_step_matches_oracle(gpu, case, Nx, Nv, order, steps):
    c = ab.Case(case, Nx, Nv, -1.0, order, fixed_body=True)
    s = ab.Solver(c, precision=64)
    o = Oracle.from_case(c)
    for _ in range(steps):
        s.cudaStep(1)
        st = o.step(1)
        cnt = s.counters()
        assert cnt["transport_flags"] == st["transport_flags"]
        assert cnt["mood_fail"] == st["mood_fail"]
        assert cnt["positivity_fixes"] == st["positivity_fixes"]
    g, m = s.cudaDownloadFull()
    assert rel(g, o.g) < 1e-10
    for q in (0, 4, 5):
        assert rel(m[:, q], o.macro[:, q]) < 1e-10, q
    assert np.abs(m[:, 1:4] - o.macro[:, 1:4]).max() < 1e-8
    np.testing.assert_array_equal(m[:, 6], o.macro[:, 6])
    assert s.cudaTotalMass() == pytest.approx(o.sum_mass(), rel=1e-12)
    s.close()


@pytest.mark.parametrize("case,Nx,Nv,order,steps", CASES[:6])
def test_fp32_step_error_against_fp64(gpu, case, Nx, Nv, order, steps):
    c = ab.Case(case, Nx, Nv, -1.0, order, fixed_body=True)
    s32 = ab.Solver(c, precision=32)
    o = Oracle.from_case(c)
    s32.cudaStep(steps)
    o.step(steps)
    g, m = s32.cudaDownloadFull()
    assert rel(m[:, 0], o.macro[:, 0]) < 5e-5
    assert rel(m[:, 4], o.macro[:, 4]) < 5e-5
    assert rel(g, o.g) < 3e-4
    s32.close()


@pytest.mark.parametrize("tag,case,Nx,Nv,order,steps,full", STEPS)
def test_gpu_matches_reference_fixtures(gpu, tag, case, Nx, Nv, order, steps, full):
    """Direct pin to the reference's own output, no oracle in between."""
    fx = golden(f"step_{tag}.npz")
    c = ab.Case(case, Nx, Nv, -1.0, order, fixed_body=True)
    s = ab.Solver(c, precision=64)
    flags = []
    for _ in range(steps):
        s.cudaStep(1)
        cnt = s.counters()
        flags.append([cnt["transport_flags"], cnt["mood_fail"]])
    np.testing.assert_array_equal(np.array(flags), fx["flags"])
    g, m = s.cudaDownloadFull()
    assert rel(m[:, 0], fx["macro"][:, 0]) < 1e-10
    assert rel(m[:, 4], fx["macro"][:, 4]) < 1e-10
    assert rel(g.sum(axis=1), fx["gsum"]) < 1e-10
    if full:
        assert rel(g, fx["g"]) < 1e-10
    s.close()


@pytest.mark.parametrize("tag,case,Nx,Nv,order,steps,full", LONG_STEPS)
def test_gpu_matches_reference_over_the_full_run(gpu, tag, case, Nx, Nv, order, steps, full):
    """The plain cavity2d (Nx 20, Nv 16, quadratic, default dt) over its 500
    steps in FP64 against the reference's own run: the same transport-flag
    and moodCheck decisions at every step, and rho, u, v, T within 1e-6
    relative (L2), the FP64 contract."""
    fx = golden(f"step_{tag}.npz")
    c = ab.Case(case, Nx, Nv, -1.0, order, fixed_body=True)
    s = ab.Solver(c, precision=64)
    flags = []
    for _ in range(steps):
        s.cudaStep(1)
        cnt = s.counters()
        flags.append([cnt["transport_flags"], cnt["mood_fail"]])
    np.testing.assert_array_equal(np.array(flags), fx["flags"])
    _, m = s.cudaDownloadFull()
    for q in (0, 1, 2, 4):
        d = np.linalg.norm(m[:, q] - fx["macro"][:, q]) / np.linalg.norm(fx["macro"][:, q])
        assert d < 1e-6, (q, d)
    s.close()


@pytest.mark.parametrize("case,Nx,Nv,order,steps", [("cavity3d", 8, 6, 2, 3),
                                                    ("cavity3d", 13, 10, 2, 3),
                                                    ("cavity3d", 9, 5, 1, 2)])
def test_lattice_march_matches_gather(gpu, case, Nx, Nv, order, steps):
    """The TMA lattice march and the coefficient gather compute the same
    transport; FP32 results agree to rounding.  The MOOD screen is off here:
    in FP32 its 1e-9 absolute slack (MLSTransport.cpp:370) sits below the
    rounding of the transported mass near a uniform state, so two summation
    orders may flag different particles."""
    c = ab.Case(case, Nx, Nv, -1.0, order)
    cfg_m = c.config(32, 0, 2)
    cfg_g = c.config(32, 0, 1)
    cfg_m.limiter = cfg_g.limiter = 0
    m = ab.Solver(c, config=cfg_m)
    g = ab.Solver(c, config=cfg_g)
    assert m.counters()["transport_kernel"] == 2
    assert g.counters()["transport_kernel"] == 1
    m.cudaStep(steps)
    g.cudaStep(steps)
    assert m.counters()["error_word"] == 0
    gm, mm = m.cudaDownloadFull()
    gg, mg = g.cudaDownloadFull()
    assert rel(gm, gg) < 1e-5
    assert rel(mm[:, 0], mg[:, 0]) < 1e-6


@pytest.mark.parametrize("case,Nx,Nv,order", [("cavity3d", 13, 10, 2), ("cavity3d", 9, 5, 2),
                                              ("cavity3d", 8, 6, 1)])
def test_packed_march_equals_scalar_march(gpu, case, Nx, Nv, order):
    """Two velocities per lane (packed fma.rn.f32x2, 64 per block) and one
    per lane give the same bits: each half of a packed FMA rounds as one
    fmaf, in the same order.  Nv = 5 has an odd row length V = 125, whose
    last lane pair straddles the end of the row."""
    c = ab.Case(case, Nx, Nv, -1.0, order)
    out = []
    for width in (2, 1):
        s = ab.Solver(c, config=c.config(32, 0, 2))
        s.set_march_width(width)
        s.cudaStep(3)
        assert s.counters()["error_word"] == 0
        out.append(s.cudaDownloadFull())
        s.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_step_is_deterministic(gpu):
    c = ab.Case("cavity3d", 12, 6, -1.0, 2)
    out = []
    for _ in range(2):
        s = ab.Solver(c, precision=32)
        s.cudaStep(5)
        out.append(s.cudaDownloadFull())
        s.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_graph_replay_matches_single_steps(gpu):
    c = ab.Case("cavity2d", 16, 12, -1.0, 2)
    a = ab.Solver(c, precision=64)
    b = ab.Solver(c, precision=64)
    a.cudaStep(6)
    for _ in range(6):
        b.cudaStep(1)
        b.sync()
    np.testing.assert_array_equal(a.cudaDownloadFull()[0], b.cudaDownloadFull()[0])


def test_mood_recollision_path(gpu):
    """A planted all-negative particle trips the transport screen and the
    post-collision moodCheck; the device takes the same branches as the
    oracle (Solver/Solver.cpp:641-646, 685-693)."""
    c = ab.Case("cavity2d", 12, 8, -1.0, 2)
    i = int(np.nonzero(c.boundary == 0)[0][20])
    c.g[i] = -50.0 * np.abs(c.g[i])
    s = ab.Solver(c, precision=64)
    o = Oracle.from_case(c)
    s.cudaStep(1)
    st = o.step(1)
    cnt = s.counters()
    assert st["mood_fail"] == 1 and cnt["mood_fail"] == 1
    assert cnt["transport_flags"] == st["transport_flags"] > 0
    g, m = s.cudaDownloadFull()
    assert rel(g, o.g) < 1e-10
    np.testing.assert_array_equal(m[:, 6], o.macro[:, 6])


def test_body_loads_match_oracle(gpu):
    c = ab.Case("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=64)
    o = Oracle.from_case(c)
    s.cudaStep(2)
    o.step(2)
    centres = c.bodies[:, 0:3]
    areas = c.bodies[:, 31]
    got = s.body_loads(centres, areas)
    want = o.body_loads(centres, areas)
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    c2 = ab.Case("cavity2d-square", 24, 8, -1.0, 2, fixed_body=True)
    s2 = ab.Solver(c2, precision=64)
    o2 = Oracle.from_case(c2)
    s2.cudaStep(2)
    o2.step(2)
    got2 = s2.body_loads(c2.bodies[:, 0:3], c2.bodies[:, 31])
    want2 = o2.body_loads(c2.bodies[:, 0:3], c2.bodies[:, 31])
    assert np.abs(got2 - want2).max() <= 1e-10 * np.abs(want2).max()


@pytest.mark.parametrize("case,Nx,Nv,precision,limiter,steps", [
    ("cavity3d", 12, 10, 64, 2, 4),
    ("cavity3d", 9, 5, 64, 2, 3),
    ("cavity3d-sphere", 12, 4, 64, 2, 2),
    ("cavity3d", 13, 10, 32, 0, 3),
])
def test_streamed_particle_kernel_matches_general(gpu, case, Nx, Nv, precision, limiter,
                                                  steps):
    """The streamed 3-D particle kernel (bulk-copied rows, post-collision
    moments from per-axis Maxwellian sums) and the general warp-per-particle
    kernel (moments summed over the written row) agree to rounding and take
    the same MOOD branches."""
    c = ab.Case(case, Nx, Nv, -1.0, 2, fixed_body=True)
    cfg_s = c.config(precision, 0, 0, 2)
    cfg_g = c.config(precision, 0, 0, 1)
    cfg_s.limiter = cfg_g.limiter = limiter
    s = ab.Solver(c, config=cfg_s)
    g = ab.Solver(c, config=cfg_g)
    assert s.counters()["particle_kernel"] == (3 if precision == 32 else 2)
    assert g.counters()["particle_kernel"] == 1
    for _ in range(steps):
        s.cudaStep(1)
        g.cudaStep(1)
        cs, cg = s.counters(), g.counters()
        assert cs["error_word"] == 0
        for k in ("transport_flags", "positivity_fixes", "mood_fail"):
            assert cs[k] == cg[k], k
    gs_, ms = s.cudaDownloadFull()
    gg, mg = g.cudaDownloadFull()
    tol = 1e-11 if precision == 64 else 1e-5
    assert rel(gs_, gg) < tol
    for q in (0, 4, 5):
        assert rel(ms[:, q], mg[:, q]) < tol, q
    assert np.abs(ms[:, 1:4] - mg[:, 1:4]).max() < (1e-8 if precision == 64 else 1e-2)
    s.close()
    g.close()


@pytest.mark.parametrize("case,Nx,Nv,steps", [("cavity3d", 13, 10, 4), ("cavity3d", 10, 8, 3),
                                              ("cavity3d", 9, 5, 3),
                                              ("cavity3d-sphere", 12, 4, 2)])
def test_row_kernels_match_streamed_particle_kernel(gpu, case, Nx, Nv, steps):
    """FP32: the three row kernels (row sums; per-particle decisions and
    tables on one thread; the collision written out) and the
    warp-per-particle streamed stage take the same MOOD and repair branches
    and agree to FP32 rounding."""
    c = ab.Case(case, Nx, Nv, -1.0, 2, fixed_body=True)
    b = ab.Solver(c, config=c.config(32, 0, 0, 2))
    w = ab.Solver(c, config=c.config(32, 0, 0, 3))
    assert b.counters()["particle_kernel"] == 3
    assert w.counters()["particle_kernel"] == 2
    for _ in range(steps):
        b.cudaStep(1)
        w.cudaStep(1)
        cb, cw = b.counters(), w.counters()
        assert cb["error_word"] == 0
        for k in ("transport_flags", "positivity_fixes", "mood_fail"):
            assert cb[k] == cw[k], k
    gb, mb = b.cudaDownloadFull()
    gw, mw = w.cudaDownloadFull()
    assert rel(gb, gw) < 1e-5
    for q in (0, 4, 5):
        assert rel(mb[:, q], mw[:, q]) < 1e-5, q
    b.close()
    w.close()


def test_row_kernels_positivity_repair(gpu):
    """FP32, planted negative nodes: the row kernels repair the same rows as
    the FP64 oracle and stay within the FP32 error of it."""
    c = ab.Case("cavity3d", 10, 6, -1.0, 2)
    inner = np.nonzero(c.boundary == 0)[0]
    for i in inner[::5]:
        c.g[i, ::4] *= -0.3
    cfg = c.config(32, 0, 0, 2)
    cfg.limiter = 0
    s = ab.Solver(c, config=cfg)
    assert s.counters()["particle_kernel"] == 3
    o = Oracle.from_case(c, limiter=0)
    for _ in range(2):
        s.cudaStep(1)
        st = o.step(1)
        assert s.counters()["positivity_fixes"] == st["positivity_fixes"]
    assert s.counters()["positivity_fixes"] > 0
    g, m = s.cudaDownloadFull()
    assert rel(g, o.g) < 3e-4
    for q in (0, 4):
        assert rel(m[:, q], o.macro[:, q]) < 5e-5, q
    s.close()


def test_streamed_particle_kernel_positivity_repair(gpu):
    """Planted negative nodes make the transported rows of many particles
    mixed-sign, so the positivity repair (MLSTransport.cpp:189-200) fires in
    the streamed kernel's separate repaired-moment pass; FP64 against the
    oracle, MOOD off so that the repaired rows are collided."""
    c = ab.Case("cavity3d", 10, 6, -1.0, 2)
    inner = np.nonzero(c.boundary == 0)[0]
    for i in inner[::5]:
        c.g[i, ::4] *= -0.3
    cfg = c.config(64, 0, 0, 2)
    cfg.limiter = 0
    s = ab.Solver(c, config=cfg)
    o = Oracle.from_case(c, limiter=0)
    for _ in range(2):
        s.cudaStep(1)
        st = o.step(1)
        cnt = s.counters()
        assert cnt["positivity_fixes"] == st["positivity_fixes"]
    assert cnt["positivity_fixes"] > 0
    g, m = s.cudaDownloadFull()
    assert rel(g, o.g) < 1e-10
    for q in (0, 4, 5):
        assert rel(m[:, q], o.macro[:, q]) < 1e-10, q
    s.close()


def test_fp32_screen_ignores_rounding_noise(gpu):
    """FP32 cannot resolve density extrema below its own rounding, so its NAD
    screen adds a floor of 64 FP32 ulps of the neighbour range to the
    reference's slack (MLSTransport.cpp:370).  Step 1, where the screen fires
    on every interior particle of the rest state, matches FP64; later FP32
    flags at most what FP64 flags, instead of the thousands of particles
    whose transported density differs from its neighbours' only by
    rounding."""
    c = ab.Case("cavity3d", 16, 10, -1.0, 2)
    s32 = ab.Solver(c, precision=32)
    s64 = ab.Solver(c, precision=64)
    for step in range(6):
        s32.cudaStep(1)
        s64.cudaStep(1)
        f32 = s32.counters()["transport_flags"]
        f64 = s64.counters()["transport_flags"]
        if step == 0:
            assert f32 == f64 == 14 ** 3
        else:
            assert f32 <= f64
    s32.close()
    s64.close()


def test_full_size_cavity3d_properties(gpu):
    """cavity3d Nx=40 Nv=10 (64 000 x 1 000): properties that hold at any
    size -- FP32 tracks FP64 on the device, the run is finite, and the mass
    bookkeeping closes: the end-of-step mass of one step is the start mass of
    the next, and the global rescale restores it after transport.

    (The lid-driven cavity's y -> L - y mirror symmetry is NOT a property of
    the reference's discretisation: its FMA-contracted wall-normal velocity
    breaks the cn = 0 ties of mirrored edge particles differently, because the
    velocity nodes fma(j, dv, vmin) are not exactly antisymmetric.)"""
    c = ab.Case("cavity3d", 40, 10, -1.0, 2)
    s32 = ab.Solver(c, precision=32)
    s64 = ab.Solver(c, precision=64)
    s32.cudaStep(3)
    s64.cudaStep(2)
    m_end = s64.counters()["mass_end"]
    s64.cudaStep(1)
    cnt = s64.counters()
    assert cnt["mass_before"] == pytest.approx(m_end, rel=1e-14)
    assert cnt["mass_after_transport"] * cnt["mass_scale"] == pytest.approx(m_end, rel=1e-14)
    g32, m32 = s32.cudaDownloadFull()
    g64, m64 = s64.cudaDownloadFull()
    assert np.isfinite(g32).all() and np.isfinite(m64).all()
    assert rel(m32[:, 0], m64[:, 0]) < 5e-5
    assert rel(g32, g64) < 1e-4
    assert s64.cudaTotalMass() == pytest.approx(cnt["mass_end"], rel=1e-14)
    s32.close()
    s64.close()
