"""The C-ABI library loads, exports every symbol include/alebgk.h declares, and
its host-only entry points and argument checks work without a GPU."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "alebgk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(alebgk_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = header_functions()
    for must in ("alebgk_upload", "alebgk_step", "alebgk_download_moments",
                 "alebgk_download_full", "alebgk_destroy", "alebgk_total_mass",
                 "alebgk_get_counters", "alebgk_body_loads"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    from alebgk4paper_b200 import _abi
    for name in header_functions():
        assert hasattr(lib, name), name
        assert name in _abi.SIGNATURES, f"{name} has no ctypes signature"


def test_create_without_device_fails_cleanly(lib):
    """With no GPU, create returns an error code and a message, never exits."""
    import torch
    if torch.cuda.is_available():
        return
    from alebgk4paper_b200 import _abi
    cfg = _abi.Config(dim=3, N=8, Nv=4, mls_order=2, precision=32, limiter=2,
                      R=208.0, tau=1e-10, vmin=-1000.0, dv=100.0, radius=1e-7)
    h = ctypes.c_void_p()
    rc = lib.alebgk_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == _abi.ECUDA
    buf = ctypes.create_string_buffer(256)
    lib.alebgk_last_error(None, buf, 256)
    assert b"device" in buf.value


def test_create_rejects_bad_config(lib):
    from alebgk4paper_b200 import _abi
    h = ctypes.c_void_p()
    bad = [dict(dim=4), dict(N=0), dict(precision=16), dict(mls_order=3),
           dict(limiter=1), dict(tau=0.0), dict(Nv=60)]
    for b in bad:
        kw = dict(dim=3, N=8, Nv=4, mls_order=2, precision=32, limiter=2, R=208.0,
                  tau=1e-10, vmin=-1000.0, dv=100.0, radius=1e-7)
        kw.update(b)
        cfg = _abi.Config(**kw)
        assert lib.alebgk_create(ctypes.byref(cfg), ctypes.byref(h)) == _abi.EINVAL, b


def test_case_build_rejects_unknown_case(lib):
    h = ctypes.c_void_p()
    assert lib.alebgk_case_build(b"cavity9d", -1, -1, -1.0, 2, 0, 1.0, ctypes.byref(h)) != 0
    assert lib.alebgk_case_build(b"7", -1, -1, -1.0, 2, 0, 1.0, ctypes.byref(h)) != 0


def test_null_arguments_are_rejected(lib):
    from alebgk4paper_b200 import _abi
    assert lib.alebgk_step(None, 1) == _abi.EINVAL
    assert lib.alebgk_sync(None) == _abi.EINVAL
    assert lib.alebgk_destroy(None) == _abi.OK
    buf = ctypes.create_string_buffer(8)
    assert lib.alebgk_last_error(None, buf, 0) == _abi.EINVAL
    m = np.zeros(7)
    assert lib.alebgk_download_moments(None, m.ctypes.data_as(_abi.c_double_p)) == _abi.EINVAL
