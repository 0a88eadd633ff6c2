"""Host logic of bench.py (no GPU): the end-to-end byte accounting, the
clock-sample summary and its throttle reasons, and the recorded peak and
traffic lookups."""
import json
import os

import bench


def test_e2e_bytes_follow_the_upload_path():
    # cavity3d Nx40 Nv10 FP32: 256 MB of FP32 rows take the host-rounding ring
    h2d, d2h, host_in = bench.e2e_bytes(64000, 1000, 1000, 32)
    assert h2d == 64000 * 1000 * 4 + 64000 * 52
    assert d2h == 64000 * 52
    assert host_in == 64000 * 1000 * 8 + 64000 * 56
    # FP64 context: the FP64 rows cross the bus
    assert bench.e2e_bytes(64000, 1000, 1000, 64)[0] == 64000 * 1000 * 8 + 64000 * 52
    # an FP32 cloud below the ring's 32 MiB copies FP64 rows too
    assert bench.e2e_bytes(1728, 1000, 1000, 32)[0] == 1728 * 1000 * 8 + 1728 * 52
    # V = 125: the FP32 device stride is 128
    n = (32 << 20) // (128 * 4)
    assert bench.e2e_bytes(n, 125, 125, 32)[0] == n * 128 * 4 + n * 52


def test_clock_summary_takes_the_median_and_the_active_reasons():
    c = bench.ClockSampler(0)
    c.lines = [
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = c.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                 "samples": 3}
    c.lines = ["0, 1500, 1965, 800, 0x8, Not Active, Active, Not Active, Not Active"]
    assert c.summary()["reasons"] == ["hw_thermal_slowdown"]
    c.lines = []
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_peak_and_traffic_come_from_the_committed_files():
    peak, src = bench.measured_peak()
    with open(os.path.join(bench.ROOT, "MEASURED_PEAKS.json")) as f:
        assert (peak, src) == (float(json.load(f)["hbm_gbs"]), "measured")
    with open(os.path.join(bench.ROOT, "profiles", "traffic.json")) as f:
        rec = json.load(f)
    for kernel in ("k_march", "k_particle_rows"):
        t, note = bench.recorded_traffic(kernel)
        assert t == rec[kernel]["bytes_per_launch"]
        assert t == rec[kernel]["dram_read_bytes"] + rec[kernel]["dram_write_bytes"]
        assert note.startswith("ncu")
    assert bench.recorded_traffic("no_such_kernel") == (None, "")
