#!/usr/bin/env python3
"""Benchmark of the B200 2D ideal-MHD + GLM step (pmhd).

Metric: zone-cycles/s (nx * ny * steps / time; one step = both SSPRK2
stages, the reference's "Mcell-steps/s", src/mhd/mhd2d_glm_gpu.cu:550-554)
on Orszag-Tang 4096 x 4096, mixed precision (binary32 reconstruction/flux/CFL,
binary64 state, recovery and update), MUSCL + SSPRK2, HLLD, CFL 0.25,
alpha 0.18.  The fp64 and fp32 builds are timed beside it at the same size,
and the relative L2 of mixed against fp64 after the same steps is reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched by torchrun, one process per GPU; every rank advances its
own full-size replica (the single-GPU path has no domain decomposition), the
timed region is bracketed by a barrier and device synchronisation, and the
slowest rank's time is used.  `--impl reference` times the reference's own
serial CPU solver (built from its sources into oracle/_ref/) on the host
cores instead; only rank 0 runs it.
"""
import argparse
import contextlib
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "precision-study_b200")
sys.path.insert(0, PKG)

METRIC = "zone-cycles/s at OT 4096²: mixed vs FP64 at stated rel-L2; % HBM roofline"
UNIT = "zone-cycles/s"
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "mhd2d_glm_cpu_fp64")
# Algorithmic HBM bytes per zone-cycle with binary64 storage: stage 1 reads
# U^n and writes U^1, stage 2 reads U^1 and U^n and writes U^{n+1}:
# 5 state passes x 9 variables x 8 bytes.  Halo re-reads are excluded.
B_ALG = {"fp64": 360, "mixed": 360, "fp32": 180}
# Per stage launch: stage 1 moves 2 passes, stage 2 moves 3; 2.5 on average.
B_ALG_PER_LAUNCH_CELL = {"fp64": 180, "mixed": 180, "fp32": 90}


def aux_steps(K):
    """Timed steps of the auxiliary Euler and Hancock lines: at least 100 (a
    20-step region of a 1-2 ms step varies by several per cent between runs),
    even (their graphs hold step pairs)."""
    k = max(K, 100)
    return k + (k & 1)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons of the
    benchmark's GPU during a marked region, from a background thread through
    NVML (read-only queries), every `interval` seconds.  Sampling starts on
    entry and goes on after mark_end() until at least one sample was taken
    after the region closed, so even a region shorter than the interval is
    bracketed.  The GPU is found by its PCI bus id (NVML numbers GPUs
    independently of CUDA_VISIBLE_DEVICES).  Where NVML cannot be opened the
    summary says so instead of giving clocks."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, gpu_index, interval=0.01, nvml=None):
        self.gpu = gpu_index
        self.interval = interval
        self.nvml = nvml  # an NVML module (tests pass a fake); None: import pynvml
        self.rows = []    # (time, sm_mhz, max_sm_mhz, reason bits)
        self.t0 = self.t1 = None
        self.error = None
        self._stop = threading.Event()
        self._thread = None
        self._handle = None
        self._lock = threading.Lock()
        self._smax = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        # The sampling thread may have been starved during a short region; a
        # sample taken here, on the caller's thread, closes the bracket.
        if self._handle is not None:
            try:
                self._sample()
            except Exception as exc:
                self.error = self.error or repr(exc)

    def _open(self):
        nv = self.nvml
        if nv is None:
            import pynvml as nv
            self.nvml = nv
        nv.nvmlInit()
        bus = None
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.gpu)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        except Exception:
            bus = None
        if bus is not None:
            try:
                self._handle = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self._handle = None
        if self._handle is None:
            self._handle = nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def _sample(self):
        nv, h = self.nvml, self._handle
        with self._lock:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            if self._smax is None:
                self._smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            try:
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except AttributeError:
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.rows.append((time.time(), float(sm), self._smax, int(bits)))

    def _run(self):
        while True:
            try:
                self._sample()
            except Exception as exc:  # a failing query ends sampling, recorded
                self.error = repr(exc)
                return
            if self._stop.is_set() and self.t1 is not None and self.rows[-1][0] > self.t1:
                return
            time.sleep(self.interval)

    def __enter__(self):
        try:
            self._open()
        except Exception as exc:
            self.error = "NVML unavailable: %r" % (exc,)
            return self
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=5)

    def summary(self):
        """Median SM clock and the throttle reasons seen during the marked
        region.  If no sample fell inside it (a region shorter than the
        interval), the samples just before and just after it stand in."""
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "samples_in_region": 0,
                    "reasons": [self.error or "no samples"]}
        t0 = self.t0 if self.t0 is not None else float("-inf")
        t1 = self.t1 if self.t1 is not None else float("inf")
        inside = [r for r in rows if t0 <= r[0] <= t1]
        used = inside
        if not used:
            before = [r for r in rows if r[0] < t0][-1:]
            after = [r for r in rows if r[0] > t1][:1]
            used = before + after
        reasons = set()
        nv = self.nvml
        for r in used:
            for name, const in self.REASONS:
                bit = getattr(nv, const, 0)
                if bit and (r[3] & bit):
                    reasons.add(name)
        sm = [r[1] for r in used]
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": used[0][2] if used else None,
               "samples": len(rows), "samples_in_region": len(inside),
               "region_s": (t1 - t0) if self.t0 is not None and self.t1 is not None else None,
               "reasons": sorted(reasons), "source": "nvml"}
        if self.error:
            out["sampler_error"] = self.error
        return out


class RankOps:
    """Barrier and max-over-ranks of a multi-process run (torch.distributed:
    one process per GPU, each advancing its own replica), or no-ops for one
    process.  device: where the reduction tensor lives ("cuda" under NCCL,
    "cpu" under gloo)."""

    def __init__(self, dist=None, device="cuda"):
        self.dist = dist
        self.device = device

    def barrier(self):
        if self.dist is None:
            return
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()
        self.dist.barrier()

    def max(self, x):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def throughput(world, cells, steps, ms):
    """Whole-job zone-cycles/s: every rank advanced `cells` for `steps` steps
    and the slowest rank took `ms`."""
    return world * cells * steps / (ms / 1e3)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(precision, n):
    """DRAM bytes per stage launch from the committed ncu summary, scaled to
    the n x n grid by cell count; None if no summary exists."""
    path = os.path.join(ROOT, "profiles", f"stage_kernel_{precision}.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        txt = f.read()
    m = re.search(r"dram_bytes_per_cell_per_launch:\s*([0-9.eE+-]+)", txt)
    return float(m.group(1)) * n * n if m else None


def run_reference_cpu(n, instances, t_end=1e-9):
    """Runs `instances` concurrent copies of the reference CPU solver on an
    n x n Orszag-Tang grid for one step (t_end below the first dt clips it)
    and returns (aggregate zone-cycles/s, per-instance walls).  Each copy's
    time is its own "Time loop wall time" line; the reference allocates its
    state arrays before that loop and allocates and copies its flux arrays
    inside every step (src/mhd/mhd2d_glm_cpu.cpp:231-250, :512-571), so one
    step times what every step costs.  Output files are suppressed by
    pointing OUTDIR at a path that cannot be created; the solver prints its
    timing before it tries to write."""
    if not os.path.exists(REF_CPU):
        return None, "reference CPU binary missing (run `make -C oracle ref` where the reference is present)"
    env = dict(os.environ, OUTDIR="/dev/null/pmhd_no_output")
    args = [REF_CPU, str(n), str(n), repr(t_end), "0.25", "muscl", "hlld", "0.18"]
    procs = [subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, env=env, text=True)
             for _ in range(instances)]
    walls = []
    for p in procs:
        out, _ = p.communicate()
        m = re.search(r"Time loop wall time = ([0-9.eE+-]+) s", out)
        s = re.search(r"Steps: (\d+)", out)
        if not m or not s or int(s.group(1)) != 1 or not float(m.group(1)) > 0.0:
            return None, "reference CPU run failed"
        walls.append(float(m.group(1)))
    return instances * n * n / max(walls), walls


# Peak host memory of one reference CPU process per cell: four ghosted state
# arrays held across the loop plus, inside a step, a copy of the state and
# the two flux arrays (7 x 9 values of 8 bytes), with margin.
REF_CPU_BYTES_PER_CELL = 9 * 8 * 8


def reference_instances(n, cap):
    """Concurrent reference processes: one per host core, at most `cap`, and
    no more than the available host memory holds at n x n."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = None
    k = min(cores, cap)
    if avail is not None:
        k = min(k, max(1, int(0.8 * avail // (REF_CPU_BYTES_PER_CELL * (n + 4) ** 2))))
    return max(1, k)


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "mhd2d_glm_gpu_{}")


def run_reference_gpu(n, reps=3, warmups=1):
    """The reference's own GPU programs (its source, recompiled unchanged for
    sm_100a into oracle/_ref/) on this GPU: Orszag-Tang n x n for 40 * 4096 / n
    steps (t_end scaled by (4096 / n)^2; 40 steps at 4096^2), timed by their
    own "Time loop wall time" line after `warmups` untimed runs, median of
    `reps` runs (the reference's perf scripts use 2 warm-ups and the median
    of 10).  The rate is taken from the line's Mcell-steps/s figure, which the
    program computes from the unrounded wall time (the seconds are printed
    with three decimals only).  Output files are suppressed as for the CPU
    baseline.  None where the binaries are absent or a run fails."""
    env = dict(os.environ, OUTDIR="/dev/null/pmhd_no_output")
    t_end = 5.5e-4 * (4096.0 / n) ** 2
    out = {}
    for prec in ("fp64", "fp32", "mixed"):
        exe = REF_GPU.format(prec)
        if not os.path.exists(exe):
            return None
        rates, walls, steps = [], [], None
        for i in range(warmups + reps):
            r = subprocess.run([exe, str(n), str(n), repr(t_end), "0.25", "muscl", "hlld", "0.18"], env=env,
                               capture_output=True, text=True, timeout=300)
            m = re.search(r"Time loop wall time = ([0-9.eE+-]+) s \(([0-9.eE+-]+) Mcell-steps/s\)", r.stdout)
            k = re.search(r"Steps: (\d+)", r.stdout)
            if not m or not k:
                return None
            rate = float(m.group(2)) * 1e6
            if not rate > 0.0:
                return None
            if i >= warmups:
                rates.append(rate)
                walls.append(float(m.group(1)))
                steps = int(k.group(1))
        out[prec] = {"value": statistics.median(rates), "unit": UNIT, "steps": steps,
                     "wall_s": statistics.median(walls), "runs": reps, "warmup_runs": warmups}
    out["note"] = ("reference src/mhd/mhd2d_glm_gpu.cu (+ _mixed.cu) compiled for sm_100a, OT "
                   f"{n}x{n}, its own time-loop clock, median of {reps} runs after {warmups} warm-up run(s)")
    return out


def bench_reference(args):
    """The reference arm: the reference's own serial CPU solver on this host,
    at the headline workload's grid (Orszag-Tang n x n, fp64; the reference
    has no CPU mixed precision).  One bench step = one reference step of the
    n x n grid.  Steps run as waves of P concurrent processes (P = host cores,
    capped by --ref-instances and by host memory), each process one step; W
    warm-up steps are one untimed wave at a small grid (binary and page cache
    warm), then ceil(K / P) timed waves.  value = zone-cycles of the timed
    waves / the sum of their wall times (each wave's wall = its slowest
    process's own time-loop clock)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    n = args.ref_n
    P = reference_instances(n, args.ref_instances)
    v, info = run_reference_cpu(256, min(P, max(1, args.warmup)))
    if v is None:
        print(json.dumps({"impl": "reference", "unavailable": info}))
        return 0
    waves = -(-args.steps // P)
    wall_sum, zc = 0.0, 0
    for _ in range(waves):
        v, walls = run_reference_cpu(n, P)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": walls}))
            return 0
        wall_sum += max(walls)
        zc += P * n * n
    value = zc / wall_sum
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (Orszag-Tang initial condition)",
        "ms_per_step": 1e3 * n * n / value,
        "config": {"workload": f"Orszag-Tang {n}x{n} fp64 (the reference CPU build has no mixed precision), "
                               "reference serial CPU solver, one process per core",
                   "nx": n, "ny": n, "instances": P, "waves": waves, "steps_run": waves * P},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": P, "kind": "reference",
                         "sample": f"{waves} wave(s) of {P} concurrent reference processes x OT {n}x{n} x 1 step; "
                                   "warm-up: one wave of OT 256x256 one-step runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def time_precision(pmhd, precision, n, warmup, steps, device, sampler=None):
    """Device-timed throughput of `steps` steps after `warmup` steps."""
    s = pmhd.Solver(nx=n, ny=n, precision=precision, device=device)
    s.init_problem(pmhd.PROBLEM_ORSZAG_TANG)
    # The sampler starts before the warm-up, so the timed steps follow the
    # warm-up steps without an idle gap.
    with (sampler if sampler is not None else contextlib.nullcontext()):
        if warmup:
            s.advance(max_steps=warmup)
        before = s.stats().kernel_launches
        if sampler is not None:
            sampler.mark_start()
        st = s.advance(max_steps=steps)
        if sampler is not None:
            sampler.mark_end()
    launches = st.kernel_launches - before
    return s, st, launches


def bench_e2e(pmhd, prec, n, W, K, device, barrier, max_over_ranks, world):
    """End to end through the C ABI: one timed region = pmhd_set_state from
    pinned host memory (interior AoS), pmhd_advance of K steps,
    pmhd_get_state back to pinned host memory; wall clock, slowest rank."""
    import numpy as np
    import torch
    dt = np.float32 if prec == "fp32" else np.float64
    s2 = pmhd.Solver(nx=n, ny=n, precision=prec, device=device)
    s2.init_problem(pmhd.PROBLEM_ORSZAG_TANG)
    host_in = torch.empty((n, n, 9), dtype=torch.float32 if dt == np.float32 else torch.float64,
                          pin_memory=True).numpy()
    host_out = torch.empty_like(torch.from_numpy(host_in)).pin_memory().numpy()
    s2.get_state(out=host_in)
    s2.advance(max_steps=W)
    barrier()
    t0 = time.perf_counter()
    s2.set_state(host_in)
    s2.advance(max_steps=K)
    s2.get_state(out=host_out)
    t1 = time.perf_counter()
    barrier()
    wall = max_over_ranks(t1 - t0)
    s2.close()
    nbytes = host_in.nbytes
    return {"value": world * n * n * K / wall, "unit": UNIT, "h2d_bytes_per_step": nbytes / K,
            "d2h_bytes_per_step": nbytes / K, "precision": prec,
            "note": "one C-ABI run per timed region: pmhd_set_state from pinned host AoS, "
                    f"pmhd_advance of {K} steps, pmhd_get_state to pinned host AoS"}


def bench_euler(pmhd, n, W, K, device, max_over_ranks, world):
    """Zone-cycles/s of the Euler sibling's 2D step (Liska-Wendroff
    configuration 3, HLLC, fused x/y sweeps) at n^2, fp64 and fp32.  A step
    reads and writes the 4 conservative planes once: 64 B/cell (fp64), 32 B
    (fp32) of algorithmic HBM traffic."""
    peak, _ = measured_peaks()
    out = {"grid": n, "problem": "Liska-Wendroff configuration 3, MUSCL-Hancock + HLLC, split x/y",
           "algorithmic_bytes_per_cell_step": {"fp64": 64, "fp32": 32}}
    for prec in ("fp64", "fp32"):
        with pmhd.Euler2D(n, config=3, precision=prec, device=device) as e:
            e.advance(max_steps=W + (W & 1))
            steps = aux_steps(K)
            st = e.advance(max_steps=steps)
            ms = max_over_ranks(st.device_ms)
            value = world * n * n * steps / (ms / 1e3)
            bpc = 64 if prec == "fp64" else 32
            gbs = bpc * n * n * steps / (ms / 1e3) / 1e9
            out[prec] = {"value": value, "unit": UNIT, "ms_per_step": ms / steps, "timed_steps": steps,
                         "roofline": {"achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}}
    return out


# Published A30 times of the reference's shock-bubble GPU program (src/euler/euler2d_cuda.cu,
# 500 x 197, 3459 steps to t = 0.0011741 s): logs/euler/compiler/gpu_default_run.log (fp64)
# and logs/euler/fp32/run.log (fp32), "Execution Time" of the time loop.
SHOCK_BUBBLE_A30_MS = {"fp64": 758.47, "fp32": 617.92}
REF_EULER_GPU = os.path.join(ROOT, "oracle", "_ref", "euler2d_gpu_{}")


def run_reference_euler_gpu(prec, reps=3, warmups=1):
    """The reference's shock-bubble GPU program (src/euler/euler2d_cuda.cu,
    recompiled unchanged for sm_100a into oracle/_ref/) on this GPU: its own
    "Execution Time" line (host clock around the time loop), median of `reps`
    runs after `warmups` untimed ones.  None where the binary is absent or a
    run fails."""
    exe = REF_EULER_GPU.format(prec)
    if not os.path.exists(exe):
        return None
    env = dict(os.environ, OUTDIR="/dev/null/pmhd_no_output")
    times, steps = [], None
    for i in range(warmups + reps):
        r = subprocess.run([exe], env=env, capture_output=True, text=True, timeout=300)
        m = re.search(r"Execution Time: ([0-9.]+) ms", r.stdout)
        k = re.search(r"Done\. Steps: (\d+)", r.stdout)
        if r.returncode != 0 or not m or not k:
            return None
        if i >= warmups:
            times.append(float(m.group(1)))
            steps = int(k.group(1))
    return {"ms": statistics.median(times), "steps": steps, "runs": reps, "warmup_runs": warmups}


def bench_shock_bubble(pmhd, device, max_over_ranks, world, reference_gpu=True):
    """The reference's shock-bubble program (Haas-Sturtevant, 500 x 197,
    MUSCL-Hancock + HLLC, split x/y, to t = 0.0011741 s: 3459 steps) run
    whole through the C ABI, fp64 and fp32, performance build: device time of
    the time loop (CUDA events around it, host polling included) and host
    wall time of pmhd_euler2d_advance, after one untimed whole run; against
    the published A30 time of the reference's GPU program and, where built,
    the same program on this GPU."""
    out = {"grid": [500, 197], "problem": "shock-bubble (src/euler/euler2d_cpu.cpp), to t = 0.0011741 s"}
    for prec in ("fp64", "fp32"):
        with pmhd.Euler2D(config="shock_bubble", precision=prec, device=device) as e:
            e.advance()
        with pmhd.Euler2D(config="shock_bubble", precision=prec, device=device) as e:
            t0 = time.perf_counter()
            st = e.advance()
            wall_ms = (time.perf_counter() - t0) * 1e3
        ms = max_over_ranks(st.device_ms)
        cells = 500 * 197 * st.steps
        rec = {"steps": st.steps, "t": st.t, "device_ms": ms, "wall_ms": wall_ms,
               "value": world * cells / (ms / 1e3), "unit": UNIT, "a30_published_ms": SHOCK_BUBBLE_A30_MS[prec],
               "a30_published_value": cells / (SHOCK_BUBBLE_A30_MS[prec] / 1e3)}
        ref = run_reference_euler_gpu(prec) if reference_gpu else None
        if ref is not None:
            rec["reference_gpu_same_box"] = ref
        out[prec] = rec
    return out


def bench_learned(pmhd, n, device, refine=4, t_end=0.25, iters=1500, every=1, max_pairs=1500, seed=11,
                  kh=False, precision="mixed", shrinks=(0.0,)):
    """Learned correction: training pairs from the solver (Orszag-Tang with
    the field scaled by B0 in {0.7, 0.85, 1.15, 1.3}; with kh, also the
    periodic Kelvin-Helmholtz double shear layer with widths {0.03, 0.045,
    0.065, 0.08}) on the n^2 coarse / (refine n)^2 fine grids, evaluation on
    the held-out B0 = 1 (and width 0.055).  Errors are relative L2 (rho, the
    mean over rho, mx, my, E, Bx, By, and all values at once) against the fine
    run restricted to the coarse grid; wall times are those of the time
    loops; the corrected run's speed-up is against the fine run's wall.  Each
    value in `shrinks` beyond the first adds a corrected run with that soft
    threshold on the network outputs (same weights)."""
    import numpy as np
    OT, KH = pmhd.PROBLEM_ORSZAG_TANG, pmhd.PROBLEM_KH_REF
    live = [0, 1, 2, 4, 5, 6]

    def err(a, ref):
        r = pmhd.relative_l2(ref, a)
        whole = float(np.sqrt(np.mean((a - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))  # all values at once
        return {"rho": float(r[0]), "mean": float(np.mean([r[k] for k in live])), "all": whole}

    train = [(OT, [b]) for b in (0.7, 0.85, 1.15, 1.3)]
    tests = {"orszag_tang_B0_1": (OT, [1.0])}
    if kh:
        train += [(KH, [w]) for w in (0.03, 0.045, 0.065, 0.08)]
        tests["kh_width_0.055"] = (KH, [0.055])
    out = {"coarse": n, "fine": refine * n, "precision": precision, "t_end": t_end, "pairs_every": every,
           "train": ("Orszag-Tang B0 in {0.7,0.85,1.15,1.3}" +
                     (" + periodic KH width in {0.03,0.045,0.065,0.08}" if kh else "")),
           "network": "4 x 3x3 conv, 32 channels, GELU, bf16 tcgen05, fp32 accumulation"}
    with pmhd.Learned(nx=n, ny=n, refine=refine, max_pairs=max_pairs, seed=seed, device=device,
                      precision=precision) as L:
        out["relax"], out["train_noise"] = L.cfg.relax, L.cfg.train_noise
        t0 = time.perf_counter()
        per_run = [L.generate(prob, par, t_end=t_end, every=every) for prob, par in train]
        t1 = time.perf_counter()
        out["pairs_per_training_run"] = per_run
        losses = L.train(iters=iters, batch=8, lr=2e-3)
        t2 = time.perf_counter()
        out.update({"pairs": L.num_pairs, "generate_s": t1 - t0, "train_s": t2 - t1, "train_iters": iters,
                    "loss_first": float(losses[:10].mean()), "loss_last": float(losses[-100:].mean())})
        for name, (prob, par) in tests.items():
            fine, sf = L.fine_run(prob, par, t_end=t_end, refine=refine)
            plain, sp = L.run(prob, par, t_end=t_end, use_net=False)
            two, s2 = L.fine_run(prob, par, t_end=t_end, refine=2)
            rec = {}
            try:
                corr, sc = L.run(prob, par, t_end=t_end, use_net=True)
            except pmhd.PmhdError as exc:  # a corrected state the solver could not advance
                rec["corrected_run"] = f"failed: {exc}"
                corr, sc = None, None
            rec["relL2_vs_fine"] = {"plain_coarse": err(plain, fine), "plain_2x": err(two, fine)}
            rec["wall_ms"] = {"fine": sf.wall_ms, "plain_coarse": sp.wall_ms, "plain_2x": s2.wall_ms}
            if corr is not None:
                rec["relL2_vs_fine"]["learned_coarse"] = err(corr, fine)
                rec["wall_ms"]["learned_coarse"] = sc.wall_ms
                rec["corrections"] = {"accepted": sc.accepted, "rejected_positivity": sc.rejected_positivity,
                                      "rejected_divergence": sc.rejected_divergence, "steps": sc.steps}
                rec["speedup_vs_fine_wall"] = sf.wall_ms / sc.wall_ms
                rec["gain"] = {k: rec["relL2_vs_fine"]["learned_coarse"][k] < rec["relL2_vs_fine"]["plain_coarse"][k]
                               for k in ("rho", "mean", "all")}
            out[name] = rec
        if len(shrinks) > 1:
            tmpdir = tempfile.TemporaryDirectory()
            path = os.path.join(tmpdir.name, "net.bin")
            L.save(path)
            for sh in shrinks[1:]:
                with pmhd.Learned(nx=n, ny=n, refine=refine, max_pairs=1, seed=seed, device=device,
                                  precision=precision, shrink=sh) as L2:
                    L2.load_weights(path)
                    for name, (prob, par) in tests.items():
                        key = f"learned_coarse_shrink_{sh:g}"
                        try:
                            corr, sc = L2.run(prob, par, t_end=t_end, use_net=True)
                            fine, _ = L.fine_run(prob, par, t_end=t_end, refine=refine)
                            out[name]["relL2_vs_fine"][key] = err(corr, fine)
                        except pmhd.PmhdError as exc:
                            out[name][key] = f"failed: {exc}"
            tmpdir.cleanup()
    return out


def bench_ensemble(pmhd, nmem, seed, prec, W, K, device, barrier, max_over_ranks, world):
    """Zone-cycles/s of the seeded uneven ensemble (square grids from
    {64,128,256,512}, half Orszag-Tang with scaled field, half Brio-Wu bands
    at a drawn slope) advanced by shared persistent launches, beside the same
    members advanced one grid at a time by the single-grid path."""
    ms_desc = pmhd.describe_ensemble(nmem, seed)
    e = pmhd.Ensemble(ms_desc, precision=prec, autotune=True, device=device)
    # Warm-up includes the autotuner (it needs a budget of >= 32 steps).
    e.advance(max_steps=max(32, W))
    barrier()
    tot = e.advance(max_steps=K)
    barrier()
    ms = max_over_ranks(tot.device_ms)
    cells = sum(m.nx * m.ny for m in ms_desc)
    # Tile height each size class runs with (the autotuner times each class).
    heights = {}
    for k, d in enumerate(ms_desc):
        heights.setdefault(str(d.nx), e.member_stats(k).tile_height)
    out = {"value": world * tot.zone_cycles / (ms / 1e3), "unit": UNIT, "members": nmem, "seed": seed,
           "cells": cells, "steps": K, "warmup_steps": max(32, W), "ms_per_step": ms / K,
           "tile_height": tot.tile_height, "tile_height_by_size": heights, "ctas": tot.ctas,
           "gpu_launches": tot.kernel_launches,
           "status": tot.status,
           "sizes": {str(s): sum(1 for m in ms_desc if m.nx == s) for s in (64, 128, 256, 512)}}
    e.close()
    # One grid at a time: the same members through pmhd_advance (same kernels,
    # one launch sequence per grid), device time summed.
    tot_ms, zc = 0.0, 0
    for d in ms_desc:
        with pmhd.Solver(nx=d.nx, ny=d.ny, gamma=d.gamma, bc=tuple(d.bc), precision=prec, device=device) as s:
            s.init_problem(d.problem, list(d.params[:d.nparams]))
            s.advance(max_steps=max(32, W))
            st = s.advance(max_steps=K)
            tot_ms += st.device_ms
            zc += st.zone_cycles
    out["one_grid_at_a_time"] = {"value": world * zc / (max_over_ranks(tot_ms) / 1e3), "unit": UNIT}
    out["speedup_vs_one_grid_at_a_time"] = out["value"] / out["one_grid_at_a_time"]["value"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "fp32"])
    ap.add_argument("--no-compare", action="store_true", help="skip the fp64/fp32 lines")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ref-n", type=int, default=4096, help="grid of one reference CPU sample")
    ap.add_argument("--ref-instances", type=int, default=64, help="max concurrent reference processes")
    ap.add_argument("--cpu-n", type=int, default=4096, help="grid of the 1-core cpu_baseline sample")
    # The auxiliary lines (ensemble, learned correction, Euler, MUSCL-Hancock)
    # are single-GPU measurements: on N > 1 ranks they default to off, so the
    # scaling runs hold their GPUs only for the headline; a value given on the
    # command line runs them on every N.
    ap.add_argument("--ensemble", type=int, default=None, help="members of the ensemble line (0: skip; 512)")
    ap.add_argument("--ensemble-seed", type=int, default=20261203)
    ap.add_argument("--learned", type=int, default=None,
                    help="coarse grid of the learned-correction line (0: skip; 512)")
    ap.add_argument("--learned-iters", type=int, default=1500, help="training iterations of the learned line")
    ap.add_argument("--euler", type=int, default=None, help="grid of the Euler-sibling line (0: skip; 4096)")
    ap.add_argument("--shock-bubble", type=int, default=1, help="whole shock-bubble runs in the Euler line (0: skip)")
    ap.add_argument("--hancock", type=int, default=None, help="grid of the MUSCL-Hancock line (0: skip; 4096)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return bench_reference(args)

    rank, world, local = dist_env()
    for name, single_gpu_default in (("ensemble", 512), ("learned", 512), ("euler", 4096), ("hancock", 4096)):
        if getattr(args, name) is None:
            setattr(args, name, single_gpu_default if world == 1 else 0)
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import numpy as np
    import pmhd

    n, K, W = args.n, args.steps, args.warmup
    prec = args.precision

    ops = RankOps(dist, "cuda")
    barrier, max_over_ranks = ops.barrier, ops.max

    # ---- headline: device-timed throughput of the chosen precision -------
    sampler = ClockSampler(local)
    barrier()
    s, st, launches = time_precision(pmhd, prec, n, W, K, local, sampler)
    barrier()
    ms = max_over_ranks(st.device_ms)
    value = throughput(world, n * n, K, ms)
    clocks = sampler.summary()
    U_main = s.get_state() if not args.no_compare else None
    s.close()

    extra = {}
    if not args.no_compare:
        for other in ("fp64", "fp32"):
            if other == prec:
                continue
            barrier()
            so, sto, _ = time_precision(pmhd, other, n, W, K, local)
            barrier()
            ms_o = max_over_ranks(sto.device_ms)
            extra[other] = {"value": world * n * n * K / (ms_o / 1e3), "ms_per_step": ms_o / K}
            if other == "fp64":
                U64 = so.get_state()
                rel = pmhd.relative_l2(U64, U_main)
                names = ["rho", "mx", "my", "mz", "E", "Bx", "By", "Bz", "psi"]
                extra["relL2_vs_fp64"] = {k: float(v) for k, v in zip(names, rel)}
                extra["relL2_vs_fp64_at"] = {"steps": W + K, "t": st.t}
                # psi starts at zero and stays at round-off level while the
                # field is still divergence-free, so its relative L2 compares
                # rounding noise with rounding noise; the field-scaled
                # difference is the meaningful figure.
                b_rms = float(np.sqrt(np.mean(U64[..., 5:8].astype(np.float64) ** 2)))
                d_psi = float(np.sqrt(np.mean((U64[..., 8].astype(np.float64) - U_main[..., 8]) ** 2)))
                extra["psi_rms_diff_over_B_rms"] = d_psi / b_rms if b_rms > 0 else None
            so.close()
        if "fp64" in extra:
            extra["speedup_vs_fp64"] = value / extra["fp64"]["value"]

    # ---- roofline of the dominant kernel (the stage kernel) -----------------
    peak, peak_kind = measured_peaks()
    stage_launches = 2 * K
    avg_launch_s = (st.device_ms / 1e3) / stage_launches  # includes graph gaps
    achieved = B_ALG_PER_LAUNCH_CELL[prec] * n * n / avg_launch_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": ncu_traffic(prec, n),
                "algorithmic_bytes_per_launch": B_ALG_PER_LAUNCH_CELL[prec] * n * n,
                "avg_launch_ms": avg_launch_s * 1e3, "kernel": "stage_kernel (stage 1 and 2 averaged)"}

    # ---- end to end through the C ABI with pinned host buffers --------------
    e2e = None
    if not args.no_e2e:
        e2e = bench_e2e(pmhd, prec, n, W, K, local, barrier, max_over_ranks, world)
        if prec != "fp64":
            # The same measurement in binary64, the precision of the reference
            # CPU arm, so an fp64-to-fp64 end-to-end comparison exists beside
            # the headline's mixed one.
            e2e["fp64"] = bench_e2e(pmhd, "fp64", n, W, K, local, barrier, max_over_ranks, world)

    # ---- ensemble: uneven grids in one persistent launch per stage -----------
    ens = None
    if args.ensemble > 0:
        ens = bench_ensemble(pmhd, args.ensemble, args.ensemble_seed, prec, W, K, local, barrier, max_over_ranks,
                             world)

    # ---- MUSCL-Hancock variant: one stage per step ----------------------------
    hancock = None
    if args.hancock > 0:
        hancock = {"grid": args.hancock, "workload": f"Orszag-Tang {args.hancock}^2, MUSCL-Hancock + HLLD + GLM",
                   "algorithmic_bytes_per_zone_cycle": {"fp64": 144, "mixed": 144, "fp32": 72}}
        U64h = None
        for hp in ("fp64", "mixed", "fp32"):
            sh = pmhd.Solver(nx=args.hancock, ny=args.hancock, precision=hp, order="hancock", device=local)
            sh.init_problem(pmhd.PROBLEM_ORSZAG_TANG)
            sh.advance(max_steps=W + (W & 1))
            sth = sh.advance(max_steps=aux_steps(K))
            msh = max_over_ranks(sth.device_ms)
            nst = aux_steps(K)
            bpc = hancock["algorithmic_bytes_per_zone_cycle"][hp]
            gbs = bpc * args.hancock ** 2 * nst / (msh / 1e3) / 1e9
            hancock[hp] = {"value": world * args.hancock ** 2 * nst / (msh / 1e3), "unit": UNIT,
                           "ms_per_step": msh / nst, "timed_steps": nst,
                           "roofline": {"achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}}
            if hp == "fp64":
                U64h = sh.get_state()
            elif hp == "mixed":
                rel = pmhd.relative_l2(U64h, sh.get_state())
                hancock["mixed"]["relL2_vs_fp64"] = {k: float(x) for k, x in
                                                     zip(["rho", "mx", "my", "mz", "E", "Bx", "By", "Bz"], rel[:8])}
                U64h = None
            sh.close()
        hancock["mixed_vs_fp64"] = hancock["mixed"]["value"] / hancock["fp64"]["value"]

    # ---- Euler sibling: fused split steps of the 2D Riemann problem ----------
    euler = None
    if args.euler > 0:
        euler = bench_euler(pmhd, args.euler, W, K, local, max_over_ranks, world)
        if args.shock_bubble:
            euler["shock_bubble"] = bench_shock_bubble(pmhd, local, max_over_ranks, world,
                                                       reference_gpu=not args.no_compare and rank == 0)

    # ---- learned coarse-grid correction: accuracy and wall time ---------------
    learned = None
    if args.learned > 0 and rank == 0:
        # The GPU test's case (64^2 coarse), then the larger configuration.
        learned = {"coarse_64": bench_learned(pmhd, 64, local, iters=args.learned_iters)}
        if args.learned >= 128:
            # BASELINE's configuration: 2048^2 fine -> 512^2 coarse, OT and KH
            # states, fine runs in binary64.
            # One pair every n / 16 coarse steps and room for 640 pairs: about 80
            # pairs from each of the eight training runs (at n / 32 and 600 the
            # four Orszag-Tang runs filled the store before any KH run).
            learned[f"coarse_{args.learned}"] = bench_learned(
                pmhd, args.learned, local, iters=1000, every=max(1, args.learned // 16), max_pairs=640, kh=True,
                precision="fp64", shrinks=(0.0, 1.0))

    # ---- CPU baseline: the reference serial solver, rank 0 at N = 1 ----------
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, info = run_reference_cpu(args.cpu_n, 1)
        if v is not None:
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"reference mhd2d_glm_cpu fp64 -O2, OT {args.cpu_n}x{args.cpu_n}, 1 step, 1 process"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": info}

    ref_gpu = None
    if world == 1 and not args.no_cpu_baseline:
        ref_gpu = run_reference_gpu(n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "f32 flux/recon/CFL + f64 state/recovery/update", "fp64": "f64",
                      "fp32": "f32"}[prec],
            "data": "synthetic (deterministic Orszag-Tang initial condition)",
            "config": {"workload": f"Orszag-Tang {n}x{n} {prec}, MUSCL+SSPRK2, HLLD eps 1e-4, CFL 0.25, alpha 0.18",
                       "nx": n, "ny": n, "precision": prec, "exact_ieee": False,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "no flush: each state array is %.2f GB > 126 MB L2" % (
                           n * n * 9 * (4 if prec == "fp32" else 8) / 1e9)},
            "roofline": roofline, "gpu_launches": launches, "clocks": clocks, "e2e": e2e,
            "cpu_baseline": cpu, "steps_run": {"t": st.t, "steps": st.steps},
        }
        line.update(extra)
        if ens is not None:
            line["ensemble"] = ens
        if learned is not None:
            line["learned"] = learned
        if euler is not None:
            line["euler2d"] = euler
        if hancock is not None:
            line["hancock"] = hancock
        if ref_gpu is not None:
            line["reference_gpu_same_box"] = ref_gpu
            line["speedup_vs_reference_gpu"] = {p: extra[p]["value"] / ref_gpu[p]["value"] if p in extra else
                                                value / ref_gpu[p]["value"] for p in ("fp64", "fp32", "mixed")
                                                if p in extra or p == prec}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
