"""Restart files in the reference's checkpoint layout (Core/Checkpoint.hpp),
host side: files written by the reference's own ckpt::save read back here
field for field, and malformed or mismatched files are refused."""
import os

import numpy as np
import pytest

from conftest import ref_available

import alebgk4paper_b200 as ab

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def _ref_case():
    from oracle.oracle import RefCase
    r = RefCase("cavity3d-cube", 12, 4, -1.0, 2, fixed_body=False)
    r.step(2)
    return r


def test_record_layout_matches_the_reference():
    from oracle.oracle import RefCase
    r = RefCase("cavity2d", 8, 6, -1.0, 2)
    assert r.checkpoint_sizes() == (56, 200, 232)


def test_reference_checkpoint_reads_back(tmp_path):
    r = _ref_case()
    path = str(tmp_path / "ref.ckpt")
    assert r.checkpoint_save(path)
    d = ab.read_checkpoint(path)
    assert d["N"] == r.N and d["gstride"] == r.gs and d["dim"] == 3 and d["step"] == 2
    assert d["t"] == pytest.approx(2 * r.dt, rel=1e-12)
    np.testing.assert_array_equal(d["g"], r.g())
    m = r.macro()
    np.testing.assert_array_equal(d["macro"][:, :6], m[:, :6])
    c = r.cloud()
    for k in ("xyz", "meshv", "wall", "boundary", "body_id"):
        np.testing.assert_array_equal(d[k], c[k], err_msg=k)
    b = r.bodies()
    np.testing.assert_array_equal(d["bodies"][:, 0:19], b[:, 0:19])
    np.testing.assert_array_equal(d["bodies"][:, 22:31], b[:, 22:31])
    assert d["body_rotates"].tolist() == [1]


def test_mismatched_or_damaged_files_are_refused(tmp_path):
    r = _ref_case()
    path = str(tmp_path / "ref.ckpt")
    assert r.checkpoint_save(path)
    with pytest.raises(ab.AlebgkError):
        ab.read_checkpoint(path, N=r.N + 1)
    with pytest.raises(ab.AlebgkError):
        ab.read_checkpoint(path, gstride=r.gs * 2)
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        data = f.read()
    cut = str(tmp_path / "cut.ckpt")
    with open(cut, "wb") as f:
        f.write(data[: size - 100])
    with pytest.raises(ab.AlebgkError):
        ab.read_checkpoint(cut)
    bad = str(tmp_path / "bad.ckpt")
    with open(bad, "wb") as f:
        f.write(b"NOTACKPT" + data[8:])
    with pytest.raises(ab.AlebgkError):
        ab.read_checkpoint(bad)
