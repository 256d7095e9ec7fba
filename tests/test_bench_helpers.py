"""bench.py's measurement helpers on the CPU: the roofline fraction's algorithmic
bytes, the traffic estimate from the committed captures, the clock summary's
parsing of nvidia-smi samples, and the peak lookup's fallback."""
import json
import os

import pytest

import bench


def test_roofline_fraction_counts_the_algorithmic_bytes(monkeypatch):
    monkeypatch.setattr(bench, "measured_hbm_peak", lambda: (1000.0, "measured"))
    # 1e6 neuron-steps x 52 B + 1e8 events x 8 B + 1e5 spikes x 8 B in 1 ms, against 1000 GB/s
    frac = bench.roofline_frac(1e6, 1e8, 1e5, 1e-3)
    assert frac == pytest.approx((52e6 + 8e8 + 8e5) / 1e-3 / 1e9 / 1000.0)


def test_profiled_traffic_scales_the_captured_ratio():
    d = json.load(open(os.path.join(bench.ROOT, "profiles", "traffic.json")))
    r = d["plain_1m/tile"]["dram_bytes_per_alg_byte"]
    assert 1.0 < r < 3.0
    assert bench.profiled_traffic("plain_1m", "tile", 5e8) == pytest.approx(r * 5e8)
    assert bench.profiled_traffic("no_such_workload", "tile", 5e8) is None


def test_clock_summary_parses_samples_and_reasons(tmp_path):
    p = tmp_path / "clocks.csv"
    p.write_text("0, 1965, 1965, 700.5, 0x0, Not Active, Not Active, Not Active, Not Active\n"
                 "0, 1950, 1965, 812.0, 0x4, Not Active, Not Active, Not Active, Active\n"
                 "0, 1965, 1965, 790.0, 0x0, Not Active, Not Active, Not Active, Not Active\n")
    cs = bench.ClockSampler(0)
    cs.path = str(p)
    s = cs.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"] and s["power_w_max"] == 812.0
    assert not p.exists()  # the sample file is removed once read


def test_clock_summary_without_samples():
    cs = bench.ClockSampler(0)
    assert cs.summary()["reasons"] == ["unsampled"]


def test_peak_falls_back_without_the_measured_file(monkeypatch, tmp_path):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_hbm_peak() == (bench.HBM_FALLBACK_GBS, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6551.0}))
    assert bench.measured_hbm_peak() == (6551.0, "measured")


def test_cpu_baseline_runs_reference_copies_on_a_small_replica():
    """The CPU baseline and the reference arm: a replica sized to the time budget,
    `copies` reference processes at once, events summed over the slowest copy."""
    from oracle import oracle
    specs, _ = bench.workload("standard_cpu", 1)
    eps, info = bench.cpu_baseline(specs[0], 20, budget_s=0.2, copies=2)
    assert eps > 0 and info["seconds"] > 0 and info["events"] > 0
    if oracle.ref_available("f32"):
        assert info["kind"] == "reference" and info["copies"] == 2
        assert eps == pytest.approx(info["events"] / info["seconds"])
    else:
        assert info["kind"] == "port" and info["copies"] == 1
    assert "replica" in info["sample"] and info["replica_synapses"] > 0


class _FakeEngine:
    """Events per cycle rising linearly for `rise` cycles, then flat (a start-up transient)."""

    class _Info:
        pass

    def __init__(self, rise, level=1000.0):
        self.t, self.ev, self.rise, self.level = 0, 0.0, rise, level

    def run(self, k):
        for _ in range(k):
            self.ev += self.level * min(1.0, self.t / self.rise)
            self.t += 1

    def info(self):
        i = self._Info()
        i.events_total = self.ev
        return i


def test_settle_waits_for_the_transient_and_stops_when_flat():
    done, per_chunk = bench.settle(_FakeEngine(4000), 3000, 10000)
    assert 4000 + 4 * 250 <= done < 10000          # past the rise by a window (3 % tolerance)
    assert per_chunk[-1] == pytest.approx(1000.0)
    done, _ = bench.settle(_FakeEngine(100), 3000, 10000)
    assert done == 3000                             # already flat: the minimum
    done, _ = bench.settle(_FakeEngine(20000), 3000, 10000)
    assert done == 10000                            # still rising: the maximum


def test_clock_sampler_polls_nvml_until_the_event_completes(monkeypatch):
    """The timed region lasts milliseconds: the sampler polls NVML between non-blocking
    queries of the end event, so every sample falls inside the region (a fake NVML and a
    fake event that completes on its fourth query)."""
    import sys
    import types
    calls = {"init": 0, "shutdown": 0}
    nv = types.SimpleNamespace(
        NVML_CLOCK_SM=0, nvmlClocksEventReasonHwSlowdown=0x8, nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlClocksEventReasonSwThermalSlowdown=0x20, nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlInit=lambda: calls.__setitem__("init", calls["init"] + 1),
        nvmlShutdown=lambda: calls.__setitem__("shutdown", calls["shutdown"] + 1),
        nvmlDeviceGetHandleByUUID=lambda u: "h", nvmlDeviceGetHandleByIndex=lambda i: "h",
        nvmlDeviceGetMaxClockInfo=lambda h, c: 1965, nvmlDeviceGetClockInfo=lambda h, c: 1950,
        nvmlDeviceGetPowerUsage=lambda h: 812000, nvmlDeviceGetCurrentClocksEventReasons=lambda h: 0x4)
    monkeypatch.setitem(sys.modules, "pynvml", nv)

    class Event:
        def __init__(self):
            self.n = 0
            self.synced = False

        def query(self):
            self.n += 1
            return self.n >= 4

        def synchronize(self):
            self.synced = True

    ev = Event()
    with bench.ClockSampler(0) as cs:
        cs.poll_until(ev, every_s=0.0)
    s = cs.summary()
    assert ev.synced and calls == {"init": 1, "shutdown": 1}
    assert s["samples"] == 4 and s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["power_w_max"] == 812.0
