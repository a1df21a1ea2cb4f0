"""Host-side pieces of bench.py that need no GPU: the clock record's summary
(median SM clock, the throttle reasons seen while timing) and the
algorithmic bytes each stage is charged in the roofline."""
import bench


def _sample(sm, mx, hw="Not Active", hw_th="Not Active", sw_th="Not Active", cap="Not Active"):
    return [str(sm), str(mx), "700.0", hw, hw_th, sw_th, cap]


def test_clock_summary_median_max_and_reasons():
    c = bench.ClockSampler(0)
    c.samples = [_sample(1965, 1965), _sample(1950, 1965, cap="Active"), _sample(1900, 1965)]
    s = c.summary()
    assert s["sm_mhz"] == 1950.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 3


def test_clock_summary_reports_every_slowdown_seen():
    c = bench.ClockSampler(0)
    c.samples = [_sample(1400, 1965, hw="Active"), _sample(1300, 1965, sw_th="Active", hw_th="Active")]
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_clock_summary_skips_unreadable_fields():
    c = bench.ClockSampler(0)
    c.samples = [_sample("[N/A]", "[N/A]"), _sample(1965, 1965)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 2


def test_clock_summary_without_samples_says_so():
    assert bench.ClockSampler(0).summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def test_stage_bytes_per_stage():
    s, a, o = 4, 1000, 300
    assert bench.stage_bytes("convolution", s, a, o, True) == 2 * 4 * 1000
    assert bench.stage_bytes("corrector", s, a, o, True) == (3 * 4 + 4) * 1000
    assert bench.stage_bytes("corrector", s, a, o, False) == 0  # isotropic: no corrector
    assert bench.stage_bytes("comparison", s, a, o, True) == 4 * (2 * 1000 + 300) + 8 * 1000
    assert bench.stage_bytes("level_set", s, a, o, True) == (4 + 4) * 1000
    assert bench.stage_bytes("redistancing", 8, a, o, True) == 2 * 8 * 1000
    assert bench.stage_bytes("end_of_step", s, a, o, True) == 0


def test_measured_peak_is_read_or_the_fallback_is_named():
    peak, kind = bench.measured_peak_hbm()
    assert peak > 0
    assert kind in ("measured", "fallback")
