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
