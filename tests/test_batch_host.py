"""Host side of the batched-cavity workload: the seeded instance list and the
longest-processing-time split over ranks."""
import math

import numpy as np

from alebgk4paper_b200.batch import CAVITY2D_VMAX, batched_cavity2d, partition_lpt


def test_instances_are_seeded_and_in_range():
    a = batched_cavity2d(96, seed=7)
    b = batched_cavity2d(96, seed=7)
    assert a == b
    assert batched_cavity2d(96, seed=8) != a
    for s in a:
        assert s["Nx"] in (24, 32, 40, 48) and s["Nv"] in (16, 20, 24)
        assert 0.5 <= s["lid_speed"] <= 10.0 and 0.5 <= s["rho0"] <= 11.0
        assert s["tau"] == 3.7142e-10 / s["rho0"]
        dx = 1e-6 / (s["Nx"] - 1)
        assert math.isclose(s["dt"] * CAVITY2D_VMAX / dx, 1.25, rel_tol=1e-15)
    # every choice appears in a batch of 96
    assert {s["Nx"] for s in a} == {24, 32, 40, 48}
    assert {s["Nv"] for s in a} == {16, 20, 24}


def test_lpt_partition_covers_every_instance_and_balances():
    specs = batched_cavity2d(96, seed=1)
    cost = [s["Nx"] ** 2 * s["Nv"] ** 2 for s in specs]
    for n in (1, 2, 4, 8):
        parts = partition_lpt(cost, n)
        assert sorted(i for p in parts for i in p) == list(range(96))
        loads = [sum(cost[i] for i in p) for p in parts]
        # LPT is within 4/3 of the optimum; the mean is a lower bound of it
        assert max(loads) <= 4.0 / 3.0 * max(np.mean(loads), max(cost)) + 1e-9
        assert partition_lpt(cost, n) == parts


def test_batch_solver_rejects_unknown_forms_before_any_device_work():
    """The graph form and the set-up mode are checked first, so a typo fails
    on the host with a clear message."""
    import pytest
    from alebgk4paper_b200.batch import BatchSolver
    with pytest.raises(ValueError, match="launch"):
        BatchSolver([], launch="cooperative")
    with pytest.raises(ValueError, match="setup"):
        BatchSolver([], setup="gpu")


def test_batch_and_launch_entry_points_are_exported():
    """The C-ABI of the batch forms, the batch autotuner and the launch
    shapes is declared in the header and exported by the library."""
    import os
    from alebgk4paper_b200 import _abi
    lib = _abi.load()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "alebgk.h")).read()
    for name in ("alebgk_batch_set_mode", "alebgk_batch_get_mode", "alebgk_batch_set_groups",
                 "alebgk_batch_autotune", "alebgk_batch_set_spin_limit", "alebgk_set_launch",
                 "alebgk_get_launch",
                 "alebgk_upload_geometry", "alebgk_set_coeff_builder"):
        assert f"{name}(" in header, name
        assert hasattr(lib, name), name
    # the batch forms are 0, 1, 2; a negative poll limit is refused
    assert lib.alebgk_batch_set_mode(None, 2) != 0
    assert lib.alebgk_batch_set_spin_limit(None, 5) != 0
    # only 0, 1, 2 are builder modes; the setting is restored
    assert lib.alebgk_set_coeff_builder(3) != 0
    assert lib.alebgk_set_coeff_builder(-1) != 0
    assert lib.alebgk_set_coeff_builder(0) == 0


def test_bench_parses_the_batch_and_error_workloads():
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "bench.py", "--help"], cwd=root, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0
    for flag in ("--batch-form", "--no-steady", "fp32-error"):
        assert flag in out.stdout, flag
