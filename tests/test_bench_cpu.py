"""Host logic of the bench that decides whether a run is kept (no GPU).

The clock record sampled during the timed region is summarised into the
median SM clock, the maximum clock and the throttle reasons seen; a run whose
record shows hw_slowdown, hw_thermal_slowdown or sw_thermal_slowdown is
re-measured, sw_power_cap is kept and noted. Also: valid-region tap counts and
the seeded synthetic image the workloads use."""
import numpy as np

import bench

HEADER_FREE_ROWS = [
    # index, sm, max sm, power, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
    "0, 1950, 1965, 990.4, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
    "0, 1965, 1965, 720.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
    "garbage line",
    "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
]


def _summary(lines, tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    with open(c.path, "w") as f:
        f.write("\n".join(lines) + "\n")
    c.proc = object()  # a sampler "ran"; summary() only reads the file
    return c.summary()


def test_clock_summary_median_and_reasons(tmp_path):
    s = _summary(HEADER_FREE_ROWS, tmp_path)
    assert s["sm_mhz"] == 1965.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_thermal_slowdown(tmp_path):
    rows = HEADER_FREE_ROWS[:1] + [
        "0, 1500, 1965, 1000.0, 0x40, Not Active, Active, Not Active, Not Active"]
    s = _summary(rows, tmp_path)
    assert "hw_thermal_slowdown" in s["reasons"]
    assert s["sm_mhz"] == (1965.0 + 1500.0) / 2


def test_clock_summary_without_sampler():
    c = bench.Clocks(0)
    c.proc = None
    assert c.summary()["reasons"] == ["nvidia-smi unavailable"]


def test_valid_taps_and_seeded_image():
    assert bench.valid_taps(4096, 4096, 31, 31) == 4066 * 4066 * 961
    assert bench.valid_taps(512, 512, 16, 16, nch=4) == 497 * 497 * 256 * 4
    a = bench.blob_field(64, 48, nblobs=5, seed=3)
    b = bench.blob_field(64, 48, nblobs=5, seed=3)
    assert a.dtype == np.float32 and a.shape == (48, 64)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, bench.blob_field(64, 48, nblobs=5, seed=4))
