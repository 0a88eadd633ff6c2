"""Field output on the host: the VTK frame, the interior diagnostics, the
timeseries row and the step line against the reference's own Core/Output.hpp
functions (compiled unmodified into oracle/_ref) on the same particles, and
the binary field dump's reader."""
import os
import struct

import numpy as np
import pytest

import alebgk4paper_b200 as ab


def _ref_case():
    from oracle.oracle import RefCase, ref_library
    if ref_library() is None:
        pytest.skip("oracle/_ref not built")
    r = RefCase("cavity3d-cube", 8, 4, -1.0, 2, fixed_body=True)
    r.step(3)
    return r


def test_vtk_frame_is_the_references_byte_for_byte(tmp_path):
    """writeVTK (Core/Output.hpp:17-51) of the reference's particles after
    three steps of cavity3d-cube, and this library's writer given the same
    positions, macros and boundary flags: the same bytes."""
    r = _ref_case()
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    r.write_vtk(ref_dir, 3, 3 * r.dt)
    want = (ref_dir / "output_000003.vtk").read_bytes()
    cl, m = r.cloud(), r.macro()
    mine = tmp_path / "mine.vtk"
    ab.write_vtk_host(mine, cl["xyz"], m, cl["boundary"], r.Nv, 3 * r.dt)
    got = mine.read_bytes()
    assert got == want
    # a frame with every section: positions, six scalars, the velocity
    assert got.count(b"SCALARS") == 6 and b"VECTORS velocity double" in got


def test_diagnostics_timeseries_and_step_line_are_the_references(tmp_path, capfd):
    r = _ref_case()
    cl, m = r.cloud(), r.macro()
    d = ab.diagnostics(m, cl["boundary"])
    want = r.diagnostics()
    for k in ("rho_avg", "KE", "T_avg", "p_avg", "mood_count", "n"):
        assert d[k] == want[k], k
    assert d["n"] == int((cl["boundary"] == 0).sum())
    # one timeseries row; the reference writes its column line on its first
    # call in the process
    ref_ts, my_ts = tmp_path / "ref.csv", tmp_path / "mine.csv"
    r.write_timeseries(ref_ts, 3 * r.dt)
    ab.write_timeseries(my_ts, 3 * r.dt, d, header=True)
    ref_lines = ref_ts.read_text().splitlines()
    my_lines = my_ts.read_text().splitlines()
    assert my_lines[-1] == ref_lines[-1]
    if len(ref_lines) == 2:
        assert my_lines == ref_lines
    ab.write_timeseries(my_ts, 4 * r.dt, d)
    assert len(my_ts.read_text().splitlines()) == 3
    # the step line (printStep, Output.hpp:111-115)
    capfd.readouterr()
    r.print_step(3, 3 * r.dt, r.dt)
    out = capfd.readouterr().out
    assert ab.format_step(3, 3 * r.dt, r.dt, d) == out


def test_vtk_writer_handles_empty_clouds_and_reports_write_errors(tmp_path):
    p = tmp_path / "empty.vtk"
    ab.write_vtk_host(p, np.zeros((0, 3)), np.zeros((0, 7)), np.zeros(0, np.int32), 4, 0.0)
    text = p.read_text()
    assert "POINTS 0 double" in text and "POINT_DATA 0" in text
    with pytest.raises(ab.AlebgkError) as e:
        ab.write_vtk_host(tmp_path / "no" / "such" / "dir.vtk", np.zeros((1, 3)),
                          np.zeros((1, 7)), np.zeros(1, np.int32), 4, 0.0)
    assert e.value.code == -6      # ALEBGK_EIO


def test_binary_field_reader(tmp_path):
    """A dump written byte by byte in the documented layout reads back; a
    wrong magic or a short file is refused."""
    n = 5
    rng = np.random.default_rng(0)
    xyz, macro = rng.normal(size=(n, 3)), rng.normal(size=(n, 7))
    boundary = np.array([0, 1, 0, 0, 1], np.int32)
    head = b"ALBGKFLD" + struct.pack("<IIQqd", 1, 3, n, 42, 1.5e-9)
    p = tmp_path / "f.bin"
    p.write_bytes(head + xyz.tobytes() + macro.tobytes() + boundary.tobytes())
    f = ab.read_fields(p)
    assert (f["step"], f["t"], f["dim"], f["N"]) == (42, 1.5e-9, 3, n)
    np.testing.assert_array_equal(f["xyz"], xyz)
    np.testing.assert_array_equal(f["macro"], macro)
    np.testing.assert_array_equal(f["boundary"], boundary)
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTFIELD" + head[8:] + xyz.tobytes())
    with pytest.raises(ab.AlebgkError):
        ab.read_fields(bad)
    short = tmp_path / "short.bin"
    short.write_bytes(head + xyz.tobytes())
    with pytest.raises(ab.AlebgkError):
        ab.read_fields(short)


def test_field_entry_points_are_exported():
    from alebgk4paper_b200 import _abi
    lib = _abi.load()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "alebgk.h")).read()
    for name in ("alebgk_vtk_write_host", "alebgk_write_vtk", "alebgk_diagnostics_host",
                 "alebgk_diagnostics", "alebgk_write_timeseries", "alebgk_format_step",
                 "alebgk_write_fields", "alebgk_read_fields"):
        assert f"{name}(" in header, name
        assert hasattr(lib, name), name
