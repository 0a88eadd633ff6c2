"""Field output from the device: the VTK frame of a stepped context against
the reference's own writeVTK after the same steps (FP64), the diagnostics,
and the binary field dump's round trip."""
import numpy as np
import pytest

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.gpu


def _numbers(text):
    return [line.split() for line in text.splitlines()]


def test_vtk_frame_of_the_device_state_matches_the_reference(gpu, tmp_path):
    """Three FP64 steps of cavity3d-cube on the device and in the reference:
    the two VTK frames have the same lines and every printed number agrees
    to its printed precision (the states agree to 1e-10, so a number may
    differ in its last printed digit where the 7-digit rounding falls
    between the two)."""
    from oracle.oracle import RefCase, ref_library
    if ref_library() is None:
        pytest.skip("oracle/_ref not built")
    r = RefCase("cavity3d-cube", 8, 4, -1.0, 2, fixed_body=True)
    r.step(3)
    c = ab.Case("cavity3d-cube", 8, 4, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=64)
    s.cudaStep(3)
    (tmp_path / "ref").mkdir()
    (tmp_path / "dev").mkdir()
    r.write_vtk(tmp_path / "ref", 3, 3 * r.dt)
    s.write_vtk(tmp_path / "dev", 3, 3 * r.dt)
    want = _numbers((tmp_path / "ref" / "output_000003.vtk").read_text())
    got = _numbers((tmp_path / "dev" / "output_000003.vtk").read_text())
    assert len(got) == len(want)
    differ = 0
    for a, b in zip(got, want):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            if x == y:
                continue
            fx, fy = float(x), float(y)       # numbers only differ in value
            differ += 1
            assert abs(fx - fy) <= 2e-6 * max(abs(fy), 1e-300) or abs(fx - fy) < 1e-290
    print(f"{differ} printed numbers differ in their last digit")
    # diagnostics of the device state against the reference's
    d, want_d = s.diagnostics(), r.diagnostics()
    assert d["n"] == want_d["n"] and d["mood_count"] == want_d["mood_count"]
    for k in ("rho_avg", "KE", "T_avg", "p_avg"):
        assert abs(d[k] - want_d[k]) <= 1e-10 * abs(want_d[k]), k
    s.close()


@pytest.mark.parametrize("precision", [32, 64])
def test_binary_field_dump_round_trip(gpu, tmp_path, precision):
    c = ab.Case("cavity2d-square", 16, 8, -1.0, 2, fixed_body=True)
    s = ab.Solver(c, precision=precision)
    s.cudaStep(2)
    p = tmp_path / "fields.bin"
    s.write_fields(p, step=2, t=2 * c.dt)
    f = ab.read_fields(p)
    assert (f["step"], f["t"], f["dim"], f["N"]) == (2, 2 * c.dt, c.dim, c.N)
    np.testing.assert_array_equal(f["macro"], s.cudaDownloadMoments())
    np.testing.assert_array_equal(f["xyz"], c.xyz)
    np.testing.assert_array_equal(f["boundary"], c.boundary)
    d = s.diagnostics()
    assert d == ab.diagnostics(f["macro"], f["boundary"])
    s.close()
