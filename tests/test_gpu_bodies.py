"""Rigid-body step on the device: surface-stress loads and the Heun
Newton-Euler update (RigidBody/BodyDynamics.cpp:17-97, 352-638), against the
compiled reference's own free-body step and against the rigid-motion
formulas."""
import numpy as np
import pytest

from conftest import golden

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu


def rodrigues(w, dt):
    """Rotation matrix of angle |w| dt about w (world frame)."""
    n = np.linalg.norm(w)
    if n < 1e-300:
        return np.eye(3)
    a = w / n
    th = n * dt
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K


@pytest.mark.parametrize("tag,case,Nx,Nv", [("cube_n12_v4_free", "cavity3d-cube", 12, 4),
                                              ("square_n24_v8_free", "cavity2d-square", 24, 8)])
def test_free_body_history_matches_reference(gpu, tag, case, Nx, Nv):
    """Eight steps of a free body in FP64 -- fluid step, Heun body step,
    geometry re-upload -- against the compiled reference's moving-body run
    (its particle count stays the same over these steps, so its cloud
    management leaves the particle set alone).  Step 1 is only rounding: the
    body starts at rest in a symmetric gas, and both codes give a velocity
    change of 1e-16 m/s, the residue of pressure forces 1e15 times larger;
    from step 2 the lid flow reaches the body and the loads are physical."""
    fx = golden(f"body_{tag}.npz")
    c = ab.Case(case, Nx, Nv, -1.0, 2, fixed_body=False)
    assert c.moving_bodies
    np.testing.assert_allclose(c.bodies, fx["bodies_before"], rtol=1e-14, atol=0)
    s = ab.Solver(c, precision=64)
    st = c.bodies.copy()
    hist = []
    for k in range(len(fx["N"])):
        assert c.N == fx["N"][k]
        s.cudaStep(1)
        st = s.body_step(st)
        c.bodies = st
        hist.append(st.copy())
        s.refresh_geometry()
    hist = np.array(hist)
    want = fx["bodies"]
    d3 = c.dim == 3
    spin = slice(7, 10) if d3 else slice(6, 7)
    torque = slice(14, 17) if d3 else slice(13, 14)
    for name, sl in (("velocity", slice(3, 6)), ("spin", spin), ("force", slice(10, 13)),
                     ("torque", torque), ("centre", slice(0, 3)),
                     ("orientation", slice(22, 31) if d3 else slice(17, 19))):
        w, g = want[1:, :, sl], hist[1:, :, sl]
        scale = np.abs(w).max()
        assert scale > 0, name
        assert np.abs(g - w).max() <= 1e-8 * scale, name
    s.close()


def _long_run(precision, steps):
    """The free cube of cavity3d-cube (Nx 12, Nv 4) for `steps` steps of
    fluid step, Heun body step and cloud management; particle counts after
    every step and the body state every 10 steps."""
    c = ab.Case("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=False)
    s = ab.Solver(c, precision=precision)
    st = c.bodies.copy()
    counts, hist = [], []
    for k in range(1, steps + 1):
        s.cudaStep(1)
        st = s.body_step(st)
        c.bodies = st
        s.refresh_geometry()
        counts.append(c.N)
        if k % 10 == 0:
            hist.append(st[0].copy())
    s.close()
    return np.array(counts), np.array(hist)


def _rotation_deg(hist, b0):
    R = hist[:, 22:31].reshape(-1, 3, 3)
    R0T = b0[22:31].reshape(3, 3).T
    return np.degrees(np.arccos(np.clip((np.einsum("kii->k", R @ R0T) - 1) / 2, -1, 1)))


def test_free_body_2000_steps_match_reference(gpu):
    """2000 steps of the free cube in FP64 against the compiled reference's
    own moving-body run: the cube moves three to four lattice steps and
    turns by 110 degrees, and the cloud management changes the particle set
    on most steps after step 254.  Every step's particle count is the
    reference's (so every removal, merge and addition decision is), and the
    body state follows the reference's to the bounds below."""
    fx = golden("body_cube_n12_v4_free_s2000.npz")
    counts, hist = _long_run(64, len(fx["N"]))
    first = int(np.argmax(counts != fx["N"])) if (counts != fx["N"]).any() else -1
    assert first < 0, f"particle count departs at step {first + 1}"
    want = fx["bodies"][:, 0]
    b0 = fx["bodies_before"][0]
    for name, sl in (("centre", slice(0, 3)), ("velocity", slice(3, 6)),
                     ("spin", slice(7, 10)), ("orientation", slice(22, 31))):
        w = want[:, sl] - (b0[sl] if name == "centre" else 0.0)
        g = hist[:, sl] - (b0[sl] if name == "centre" else 0.0)
        err = np.abs(g - w).max() / np.abs(w).max()
        print(f"FP64 free cube, 2000 steps: {name} max error {err:.2e} of its range")
        assert err < 1e-6, name
    rot, rot_ref = _rotation_deg(hist, b0)[-1], _rotation_deg(want, b0)[-1]
    print(f"rotation after 2000 steps: {rot:.6f} deg (reference {rot_ref:.6f})")
    assert abs(rot - rot_ref) <= 1e-6 * rot_ref


def test_body_step_rigid_motion_and_wall_state(gpu):
    """A cube given a velocity and a spin: its surface particles move by the
    rigid motion of the old state (Rodrigues rotation about the old angular
    velocity, then translation), the orientation turns by the same rotation,
    and every surface particle's stored wall state becomes the face normal
    and U_w = V + w x r of the new state, with the mesh velocity = U_w."""
    c = ab.Case("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=False)
    s = ab.Solver(c, precision=64)
    s.cudaStep(1)
    st = c.bodies.copy()
    v0 = np.array([3.0, -2.0, 1.0])
    w0 = np.array([2.0e7, -1.0e7, 3.0e7])
    st[0, 3:6] = v0
    st[0, 7:10] = w0
    st[0, 6] = w0[2]
    dt = c.dt
    xyz0, _, _ = s.download_geometry()
    surf = np.nonzero((c.boundary != 0) & (c.body_id >= 0))[0]
    got = s.body_step(st, dt)
    xyz1, mv1, wall1 = s.download_geometry()
    cen0 = st[0, 0:3]
    Rw = rodrigues(w0, dt)
    r0 = xyz0[surf] - cen0
    want_xyz = cen0 + dt * v0 + r0 @ Rw.T
    np.testing.assert_allclose(xyz1[surf], want_xyz, rtol=0, atol=1e-20)
    np.testing.assert_allclose(got[0, 0:3], cen0 + dt * v0, rtol=1e-15, atol=0)
    Rm0 = st[0, 22:31].reshape(3, 3)
    Rm1 = got[0, 22:31].reshape(3, 3)
    np.testing.assert_allclose(Rm1, Rw @ Rm0, atol=1e-12)
    np.testing.assert_allclose(Rm1 @ Rm1.T, np.eye(3), atol=1e-14)
    v1, w1 = got[0, 3:6], got[0, 7:10]
    r1 = xyz1[surf] - got[0, 0:3]
    np.testing.assert_allclose(wall1[surf, 3:6], v1 + np.cross(w1, r1), rtol=1e-12,
                               atol=1e-12 * np.abs(v1).max())
    np.testing.assert_array_equal(mv1[surf], wall1[surf, 3:6])
    n = wall1[surf, 0:3]
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0, rtol=1e-14)
    # each normal is a face normal of the rotated cube, pointing outward
    body = r1 @ Rm1                                  # body-frame coordinates
    f = np.argmax(np.abs(body), axis=1)
    sign = np.sign(body[np.arange(len(surf)), f])
    np.testing.assert_allclose(n, sign[:, None] * Rm1[:, f].T, atol=1e-14)
    # fluid particles are untouched
    fluid = np.setdiff1d(np.arange(c.N), surf)
    np.testing.assert_array_equal(xyz1[fluid], xyz0[fluid])
    s.close()


def test_body_step_wall_contact(gpu):
    """A cube pushed through the x = L wall is shifted back to 0.4 dx inside
    it as one rigid body, and its velocity into the wall is removed
    (BodyDynamics.cpp:519-590)."""
    c = ab.Case("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=False)
    s = ab.Solver(c, precision=64)
    s.cudaStep(1)
    st = c.bodies.copy()
    p = c.params
    xhi = max(p["xleft"], p["xright"])
    xyz0, _, _ = s.download_geometry()
    surf = np.nonzero((c.boundary != 0) & (c.body_id >= 0))[0]
    reach = xyz0[surf, 0].max() - st[0, 0]
    dt = c.dt
    # velocity that carries the surface 2 dx past the wall in one step
    vx = (xhi - (st[0, 0] + reach) + 2 * p["dx"]) / dt
    st[0, 3:6] = [vx, 0.5, 0.0]
    got = s.body_step(st, dt)
    xyz1, _, _ = s.download_geometry()
    assert xyz1[surf, 0].max() == pytest.approx(xhi - 0.4 * abs(p["dx"]), rel=1e-12)
    assert got[0, 3] == 0.0
    assert got[0, 4] != 0.0                           # tangential motion kept
    shift = xyz1[surf] - xyz0[surf]
    np.testing.assert_allclose(shift - shift[0], 0.0, atol=1e-21)
    s.close()


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("case,Nx,Nv,v,w", [
    ("cavity3d-cube", 12, 4, (300.0, 0.0, 150.0), (0.0, 2.0e9, 0.0)),
    ("cavity2d-square", 24, 8, (400.0, 200.0, 0.0), (0.0, 0.0, 3.0e9))])
def test_geometry_refresh_in_place_equals_full_upload(gpu, precision, case, Nx, Nv, v, w):
    """The geometry refresh of a body step builds the stencil classes and
    slot lists on the device from the uploaded geometry, solves the tables
    there, and keeps the distribution where it is.  Over body steps it gives
    bitwise the state of the full re-upload with the host class builder and
    host tables (the slot order fixes the transport's summation order, so any
    difference in the slot lists would show)."""
    from alebgk4paper_b200 import _abi
    lib = _abi.load()
    out = []
    # 0: device classes and tables; 1: host; 2: host classes with device
    # tables, the path a hash collision of two stencil keys takes
    for builder in (0, 1, 2):
        lib.alebgk_set_coeff_builder(builder)
        try:
            c = ab.Case(case, Nx, Nv, -1.0, 2, fixed_body=False)
            st = c.bodies.copy()
            st[0, 3:6] = v
            if case.startswith("cavity3d"):
                st[0, 7:10] = w
            else:
                st[0, 6] = w[2]
            c.bodies = st
            s = ab.Solver(c, precision=precision)
            for _ in range(4):
                s.cudaStep(1)
                st = s.body_step(st)
                c.bodies = st
                s.refresh_geometry()
            s.cudaStep(1)
            out.append((s.cudaDownloadFull(), st.copy(), c.N))
            s.close()
        finally:
            lib.alebgk_set_coeff_builder(0)
    (g0, m0), st0, n0 = out[0]
    for (g1, m1), st1, n1 in out[1:]:
        assert n0 == n1
        np.testing.assert_array_equal(g0, g1)
        np.testing.assert_array_equal(m0, m1)
        np.testing.assert_array_equal(st0, st1)
