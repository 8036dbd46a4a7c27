"""Host helpers of bench.py on CPU: the clock sampler's parsing of
nvidia-smi samples (only samples inside the timed region count; throttle
reasons are reported), the step count of the auxiliary lines, and the
traffic figure read from the committed ncu summary."""
import datetime
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _line(ts, sm, power_cap="Not Active", thermal="Not Active"):
    stamp = datetime.datetime.fromtimestamp(ts).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return f"{stamp}, 0, {sm}, 1965, 700.0, 0x0, Not Active, Not Active, {thermal}, {power_cap}\n"


def test_clock_sampler_keeps_samples_inside_the_region():
    s = bench.ClockSampler(0)
    s.proc = object()  # as if nvidia-smi had started
    s.out = tempfile.TemporaryFile(mode="w+")
    t0 = 1_800_000_000.0
    s.out.write(_line(t0 - 0.2, 120))                           # idle, before the region
    s.out.write(_line(t0 + 0.05, 1965))
    s.out.write(_line(t0 + 0.10, 1950, power_cap="Active"))
    s.out.write(_line(t0 + 0.40, 1965, thermal="Active"))       # after the region
    s.t0, s.t1 = t0, t0 + 0.2
    r = s.summary()
    assert r["samples"] == 2 and r["samples_in_region"] == 2
    assert r["sm_mhz"] == (1965 + 1950) / 2 and r["sm_max_mhz"] == 1965
    assert r["reasons"] == ["sw_power_cap"]


def test_clock_sampler_short_region_takes_the_next_sample():
    s = bench.ClockSampler(0)
    s.proc = object()
    s.out = tempfile.TemporaryFile(mode="w+")
    t0 = 1_800_000_000.0
    s.out.write(_line(t0 - 0.1, 120))
    s.out.write(_line(t0 + 0.09, 1965))
    s.t0, s.t1 = t0, t0 + 0.05
    r = s.summary()
    assert r["samples"] == 1 and r["samples_in_region"] == 0 and r["sm_mhz"] == 1965


def test_auxiliary_lines_time_at_least_100_even_steps():
    assert bench.aux_steps(20) == 100
    assert bench.aux_steps(101) == 102
    assert bench.aux_steps(200) == 200


def test_traffic_comes_from_the_committed_profile():
    t = bench.ncu_traffic("mixed", 1000)
    assert t is not None and 150.0 * 1e6 < t < 200.0 * 1e6  # ~171 B per cell per launch


def test_reference_gpu_rates_are_parsed_from_its_stdout(tmp_path, monkeypatch):
    """run_reference_gpu reads the reference program's own "Done. Steps" and
    "Time loop wall time" lines (fake programs here print them)."""
    for prec, wall in (("fp64", "0.902"), ("fp32", "0.494"), ("mixed", "0.876")):
        exe = tmp_path / f"mhd2d_glm_gpu_{prec}"
        exe.write_text("#!/bin/sh\n"
                       "echo 'Done. Steps: 40, final t = 0.00055'\n"
                       f"echo 'Time loop wall time = {wall} s (744.09 Mcell-steps/s)'\n"
                       "exit 5\n")
        exe.chmod(0o755)
    monkeypatch.setattr(bench, "REF_GPU", str(tmp_path / "mhd2d_glm_gpu_{}"))
    r = bench.run_reference_gpu(64)
    assert r["fp64"]["steps"] == 40 and r["fp64"]["value"] == 64 * 64 * 40 / 0.902
    assert r["mixed"]["wall_s"] == 0.876


def test_reference_gpu_absent_gives_none(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "REF_GPU", str(tmp_path / "missing_{}"))
    assert bench.run_reference_gpu(64) is None
