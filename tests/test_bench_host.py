"""Host helpers of bench.py on CPU: the clock sampler (NVML samples, here
from a fake: only samples inside the timed region count, throttle reasons
are reported, the sampling thread brackets short regions), the step count of
the auxiliary lines, the traffic figure read from the committed ncu summary,
and the parsing of the reference programs' timing lines."""
import os
import sys
import threading

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class FakeNvml:
    """Stands in for the NVML bindings: clocks and reason bits from a script
    of (sm_mhz, reason bits) samples, the last one repeated."""
    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonSwPowerCap = 0x4
    nvmlClocksEventReasonHwPowerBrakeSlowdown = 0x80

    def __init__(self, script):
        self.script = list(script)
        self.i = 0
        self.lock = threading.Lock()

    def nvmlInit(self):
        pass

    def nvmlDeviceGetHandleByPciBusId(self, bus):
        return "gpu"

    def nvmlDeviceGetHandleByIndex(self, i):
        return "gpu"

    def _cur(self):
        return self.script[min(self.i, len(self.script) - 1)]

    def nvmlDeviceGetClockInfo(self, h, kind):
        return self._cur()[0]

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        with self.lock:
            v = self._cur()[1]
            self.i += 1
        return v


def test_clock_sampler_keeps_samples_inside_the_region():
    s = bench.ClockSampler(0, nvml=FakeNvml([]))
    t0 = 1_800_000_000.0
    s.rows = [(t0 - 0.2, 120.0, 1965.0, 0),          # idle, before the region
              (t0 + 0.05, 1965.0, 1965.0, 0),
              (t0 + 0.10, 1950.0, 1965.0, 0x4),      # sw_power_cap
              (t0 + 0.40, 1965.0, 1965.0, 0x40)]     # thermal, after the region
    s.t0, s.t1 = t0, t0 + 0.2
    r = s.summary()
    assert r["samples"] == 4 and r["samples_in_region"] == 2
    assert r["sm_mhz"] == (1965 + 1950) / 2 and r["sm_max_mhz"] == 1965
    assert r["reasons"] == ["sw_power_cap"]


def test_clock_sampler_short_region_uses_the_neighbouring_samples():
    s = bench.ClockSampler(0, nvml=FakeNvml([]))
    t0 = 1_800_000_000.0
    s.rows = [(t0 - 0.01, 1960.0, 1965.0, 0), (t0 + 0.09, 1965.0, 1965.0, 0x8)]
    s.t0, s.t1 = t0, t0 + 0.05
    r = s.summary()
    assert r["samples_in_region"] == 0 and r["sm_mhz"] == (1960 + 1965) / 2
    assert r["reasons"] == ["hw_slowdown"]


def test_clock_sampler_thread_samples_through_the_region():
    """The thread samples from entry and stops only after a sample taken
    once the region closed, so a short region still has samples in it."""
    fake = FakeNvml([(1965, 0)] * 3 + [(1900, 0x4)])
    s = bench.ClockSampler(0, interval=0.002, nvml=fake)
    with s:
        s.mark_start()
        import time
        time.sleep(0.05)
        s.mark_end()
    r = s.summary()
    assert r["samples_in_region"] >= 1
    assert s.rows[-1][0] > s.t1
    assert r["sm_max_mhz"] == 1965


def test_clock_sampler_without_nvml_reports_why():
    class Broken:
        def nvmlInit(self):
            raise OSError("no driver")
    s = bench.ClockSampler(0, nvml=Broken())
    with s:
        s.mark_start()
        s.mark_end()
    r = s.summary()
    assert r["sm_mhz"] is None and r["samples"] == 0 and "no driver" in r["reasons"][0]


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
        rate = "%.2f" % (64 * 64 * 40 / float(wall) / 1e6)
        exe.write_text("#!/bin/sh\n"
                       "echo 'Done. Steps: 40, final t = 0.00055'\n"
                       f"echo 'Time loop wall time = {wall} s ({rate} Mcell-steps/s)'\n"
                       "exit 5\n")
        exe.chmod(0o755)
    monkeypatch.setattr(bench, "REF_GPU", str(tmp_path / "mhd2d_glm_gpu_{}"))
    r = bench.run_reference_gpu(64)
    assert r["fp64"]["steps"] == 40 and abs(r["fp64"]["value"] - 64 * 64 * 40 / 0.902) < 1e4
    assert r["mixed"]["wall_s"] == 0.876 and r["mixed"]["runs"] == 3


def test_reference_gpu_zero_wall_gives_none(tmp_path, monkeypatch):
    """A run too short for the printed wall time (0.000 s, 0.00 Mcell-steps/s)
    yields no rate instead of a division by zero."""
    for prec in ("fp64", "fp32", "mixed"):
        exe = tmp_path / f"mhd2d_glm_gpu_{prec}"
        exe.write_text("#!/bin/sh\necho 'Done. Steps: 2, final t = 1e-06'\n"
                       "echo 'Time loop wall time = 0.000 s (inf Mcell-steps/s)'\n")
        exe.chmod(0o755)
    monkeypatch.setattr(bench, "REF_GPU", str(tmp_path / "mhd2d_glm_gpu_{}"))
    assert bench.run_reference_gpu(64) is None


def test_reference_gpu_absent_gives_none(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "REF_GPU", str(tmp_path / "missing_{}"))
    assert bench.run_reference_gpu(64) is None


def test_reference_shock_bubble_time_is_parsed_from_its_stdout(tmp_path, monkeypatch):
    """run_reference_euler_gpu reads the shock-bubble GPU program's own "Done.
    Steps" and "Execution Time" lines (a fake program prints them; the median
    of the timed runs after the warm-up is kept)."""
    times = tmp_path / "times"
    times.write_text("900.0\n330.0\n320.0\n340.0\n")
    exe = tmp_path / "euler2d_gpu_fp64"
    exe.write_text("#!/bin/sh\n"
                   f"t=$(head -1 {times}); sed -i 1d {times}\n"
                   "echo 'Done. Steps: 3459'\n"
                   "echo \"Execution Time: $t ms (0.3 s)\"\n")
    exe.chmod(0o755)
    monkeypatch.setattr(bench, "REF_EULER_GPU", str(tmp_path / "euler2d_gpu_{}"))
    r = bench.run_reference_euler_gpu("fp64")
    assert r == {"ms": 330.0, "steps": 3459, "runs": 3, "warmup_runs": 1}
    assert bench.run_reference_euler_gpu("fp32") is None  # no such program


def test_reference_shock_bubble_failure_gives_none(tmp_path, monkeypatch):
    exe = tmp_path / "euler2d_gpu_fp64"
    exe.write_text("#!/bin/sh\necho 'CUDA Error at x:1 - no device'\nexit 1\n")
    exe.chmod(0o755)
    monkeypatch.setattr(bench, "REF_EULER_GPU", str(tmp_path / "euler2d_gpu_{}"))
    assert bench.run_reference_euler_gpu("fp64") is None
