"""Host logic of bench.py that needs no GPU: the seeded input generators, the metric
arithmetic, the roofline denominator's source, and the clock sampler's reading of NVML
clock-event reasons (against a fake NVML)."""
import json

import numpy as np

import bench

M64 = (1 << 64) - 1


def splitmix64_sequential(seed, stream, n):
    """SplitMix64 (Steele, Lea & Flood 2014) as a sequential generator: state += GAMMA, then
    the output mix; started at mix(seed << 8 | stream)."""
    def mix(z):
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9 & M64
        z = (z ^ (z >> 27)) * 0x94D049BB133111EB & M64
        return z ^ (z >> 31)
    state = mix(((seed << 8) | stream) & M64)
    out = []
    for _ in range(n):
        state = (state + bench.GAMMA) & M64
        out.append(mix(state))
    return out


def test_splitmix64_is_the_sequential_generator_in_any_chunking():
    ref = splitmix64_sequential(0, 0, 300)
    assert bench.splitmix64(0, 0, 300).tolist() == ref
    assert bench.splitmix64(0, 0, 300, chunk=7).tolist() == ref
    assert bench.splitmix64(0, 0, 100, start=200).tolist() == ref[200:]
    assert bench.splitmix64(3, 5, 10).tolist() == splitmix64_sequential(3, 5, 10)


def test_workload_inputs_have_their_stated_ranges():
    k, v = bench.gen_inputs("sort_by_key_u32", 1 << 16)
    assert k.dtype == np.uint32 and v.tolist() == list(range(1 << 16))
    assert k.max() > (1 << 31) and len(np.unique(k)) > (1 << 16) - 10  # full 32-bit range
    x, _ = bench.gen_inputs("inclusive_scan_i32", 1 << 16)
    assert x.dtype == np.int32 and x.min() == -1000 and x.max() == 1000
    f, _ = bench.gen_inputs("reduce_f32", 1 << 16)
    assert f.dtype == np.float32 and f.min() >= 0.0 and f.max() < 1.0
    lens = bench.segment_lengths(100_000)
    assert lens.min() >= 1 and lens.max() <= (1 << 20) and 200 <= np.median(lens) <= 320


def test_metric_arithmetic():
    assert bench.units_per_s_to_metric("sort_by_key_u32", 2 * 10**9, 2.0) == 1.0  # Gkeys/s
    assert bench.units_per_s_to_metric("inclusive_scan_i32", 10**9, 1.0) == 8.0  # GB/s at 8 B/elem
    assert bench.units_per_s_to_metric("reduce_f32", 10**9, 2.0) == 2.0
    assert bench.units_per_s_to_metric("serving_c5", 500, 0.25) == 2000.0
    assert bench.replica_rate(100, 4, 2.0) == 200.0  # all ranks' units over the slowest rank's time


def test_roofline_denominator_source(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peak() == (bench.HBM_FALLBACK_GBS, "of fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6455.6}))
    assert bench.measured_peak() == (6455.6, "of measured")


class FakeNvml:
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, reasons):
        self.clocks, self.reasons = list(clocks), list(reasons)

    def nvmlDeviceGetClockInfo(self, h, kind):
        return self.clocks.pop(0) if len(self.clocks) > 1 else self.clocks[0]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons.pop(0) if len(self.reasons) > 1 else self.reasons[0]


def sampler_with(nv, max_mhz=1965):
    s = bench.ClockSampler.__new__(bench.ClockSampler)
    s.samples, s.reasons, s.ok, s.period, s.max_mhz = [], set(), True, 0.001, max_mhz
    s.nv, s.h = nv, object()
    return s


def test_clock_sampler_reports_median_clock_and_every_reason_seen():
    import time
    s = sampler_with(FakeNvml([1965, 1900, 1965], [0x0, 0x4, 0x8 | 0x20, 0x0]))
    with s:
        time.sleep(0.05)
    out = s.summary()
    assert out["sm_max_mhz"] == 1965 and out["sm_mhz"] == 1965 and out["samples"] >= 4
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap", "sw_thermal_slowdown"]


def test_clock_sampler_without_nvml():
    s = bench.ClockSampler.__new__(bench.ClockSampler)
    s.ok = False
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
