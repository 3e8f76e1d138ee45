"""Host-side pieces of bench.py's measurement contract, on CPU: the clock record (median SM clock
under load, throttle reasons, only samples inside the timed region), the HBM peak lookup, and
the defaults of a flagless run."""
import sys

import pytest

import bench


class _DoneProcess:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sample(sm, sm_max=1965, reasons=("Not Active",) * 4):
    return ", ".join(["0", str(sm), str(sm_max), "612.4", "0x0000000000000000", *reasons])


def _sampler(lines, first):
    c = bench.ClockSampler(0)
    c.proc = _DoneProcess()
    c.lines = list(lines)
    c.first = first
    return c


def test_clock_record_keeps_only_samples_inside_the_timed_region():
    # a pre-roll sample at a low clock is ignored; the median of the in-region samples is reported
    lines = [_sample(900), _sample(1965), _sample(1950), _sample(1965)]
    rec = _sampler(lines, first=1).stop()
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["samples"] == 3 and rec["samples_in_timed_region"] == 3
    assert rec["reasons"] == []


def test_clock_record_reports_throttle_reasons():
    hot = ("Not Active", "Active", "Not Active", "Active")  # hw_thermal_slowdown, sw_power_cap
    rec = _sampler([_sample(1965), _sample(1500, reasons=hot)], first=0).stop()
    assert rec["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert rec["sm_mhz"] == pytest.approx((1965 + 1500) / 2)


def test_short_timed_region_falls_back_to_the_sample_just_before_it():
    rec = _sampler([_sample(1965)], first=1).stop()
    assert rec["samples"] == 1 and rec["samples_in_timed_region"] == 0
    assert rec["sm_mhz"] == 1965.0


def test_clock_record_without_nvidia_smi():
    c = bench.ClockSampler(0)
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_malformed_lines_are_skipped():
    rec = _sampler(["[Unknown Error]", _sample(1965), "0, N/A, N/A"], first=0).stop()
    assert rec["samples"] == 1 and rec["sm_mhz"] == 1965.0


def test_peak_lookup_is_positive_and_labelled():
    gbs, kind = bench.peaks()
    assert gbs > 0 and kind in ("measured", "fallback")


def test_flagless_run_defaults(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.impl, a.warmup) == (1, "ours", 3)
    assert a.steps >= 1 and a.warmup >= 3
    assert a.eliminated == bench.L_FULL


def test_reference_arm_times_the_stated_workload_without_scaling(monkeypatch, capsys):
    """The reference arm runs the reference library on the same workload dict as the device arm
    (here shrunk to L=3,000 eliminated blocks to stay fast on CPU), each timed step at full size
    of that workload, the value the mean of the steps, with no sample scaling."""
    import json

    import oracle
    if not oracle.available("ref"):
        pytest.skip("reference library not built")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                                      "--eliminated", "3000"])
    monkeypatch.delenv("RANK", raising=False)
    a = bench.parse()
    bench.run_reference(a)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["config"] == bench.config_dict(1, 3000)
    assert line["converged"] and len(line["iterations"]) == 2
    lo, med, hi = line["step_ms_min_median_max"]
    assert lo <= line["value"] <= hi and line["value"] == line["ms_per_step"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 1
    assert "scaled" not in line["cpu_baseline"]["sample"]
    assert line["e2e"]["value"] == line["value"]
