"""Host-side helpers of bench.py that decide whether a timed run counts: the
clock record taken during the timed region (median SM clock, maximum, and
which throttle reasons were active) and the core count of the CPU
baseline.  No GPU: the sampler's CSV is written here as nvidia-smi writes
it (clocks.sm, clocks.max.sm, power.draw, hw_slowdown, hw_thermal_slowdown,
sw_thermal_slowdown, sw_power_cap; csv, noheader, nounits)."""
import tempfile

import bench


def _summary(lines):
    s = bench.ClockSampler(0)
    s.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    s.file.write("".join(line + "\n" for line in lines))
    s.file.flush()
    return s.summary()


def test_clean_record():
    r = _summary(["1965, 1965, 640.1, Not Active, Not Active, Not Active, Not Active"] * 3 +
                 ["1950, 1965, 700.0, Not Active, Not Active, Not Active, Not Active"])
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == [] and r["samples"] == 4


def test_power_cap_and_thermal_reasons_are_reported():
    r = _summary(["1320, 1965, 998.0, Not Active, Not Active, Not Active, Active",
                  "1305, 1965, 999.5, Not Active, Not Active, Active, Active",
                  "1330, 1965, 997.0, Not Active, Not Active, Not Active, Active"])
    assert r["sm_mhz"] == 1320.0
    assert r["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]


def test_malformed_rows_are_skipped_and_empty_record_is_unsampled():
    r = _summary(["[N/A], 1965, 500.0, Not Active, Not Active, Not Active, Not Active",
                  "1965, 1965, 500.0, Not Active, Not Active, Not Active, Not Active",
                  "garbage"])
    assert r["sm_mhz"] == 1965.0 and r["samples"] == 2
    assert _summary([]) == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def test_physical_cores():
    assert bench.physical_cores() >= 1
