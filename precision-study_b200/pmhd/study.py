"""Precision study driver and .dat comparison.

    python -m pmhd.study compare FP64.dat OTHER.dat
        Per-variable L1 / L2(RMS) / Linf / relL2 table of two .dat files,
        same definitions and layout detection as the reference's
        analysis/mhd/compare_precision.py (relL2 = RMS(a - b) / RMS(a)).

    python -m pmhd.study run --n 1024 --t-end 0.5 [--problem ot|kh_reflect]
                             [--runs fp64,fp64_exact,fp32,mixed]
        Runs the same problem in fp64 (FMA), fp64 (exact IEEE, no FMA),
        fp32 and mixed on one GPU (or the listed subset; fp64 always runs)
        and prints one JSON object: zone-cycles/s of each, and the relative L2
        of every other run against fp64 per conserved variable and per .dat
        primitive column.  The exact-vs-FMA fp64 pair is the rounding noise
        floor the mixed result is measured against.

    python -m pmhd.study conv --batch 8 --n 512 [--reps 20]
        Times one layer of the learned correction's network (pmhd_conv3x3,
        GELU, 32 -> 32 channels, bf16 NHWC images, tcgen05) on seeded data:
        microseconds per call (CUDA events around each call, which includes
        the call's own stream synchronisation), its FLOP rate and the
        algorithmic HBM bytes (input read once, z and gelu(z) written).
"""
import argparse
import json
import sys
import time

import numpy as np

from . import (LAYOUT_INTERIOR, PROBLEM_KH_REFLECT, PROBLEM_ORSZAG_TANG, Solver, conserved_to_dat_columns,
               relative_l2)

DAT_NAMES = ["rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "E"]
CONS_NAMES = ["rho", "mx", "my", "mz", "E", "Bx", "By", "Bz", "psi"]


def compare_dat(path_a, path_b, out=sys.stdout):
    a = np.loadtxt(path_a)
    b = np.loadtxt(path_b)
    if a.shape != b.shape:
        raise SystemExit(f"ERROR: shape mismatch {a.shape} vs {b.shape}")
    ncol = a.shape[1]
    if ncol == 10:
        cols, layout = list(range(1, 10)), "1D Brio-Wu"
    elif ncol == 13:
        cols, layout = list(range(2, 11)), "2D OT-GLM"
    else:
        raise SystemExit(f"ERROR: unknown layout, ncol={ncol}")
    print(f"# layout = {layout}   N = {a.shape[0]}   cols = {ncol}", file=out)
    print(f"{'var':>4} {'L1':>12} {'L2(RMS)':>12} {'Linf':>12} {'relL2':>10}", file=out)
    print("-" * 56, file=out)
    res = {}
    for nm, c in zip(DAT_NAMES, cols):
        d = a[:, c] - b[:, c]
        l1, l2, linf = np.mean(np.abs(d)), np.sqrt(np.mean(d * d)), np.max(np.abs(d))
        ref = np.sqrt(np.mean(a[:, c] ** 2))
        rel = l2 / ref if ref > 0 else 0.0
        res[nm] = {"L1": l1, "L2": l2, "Linf": linf, "relL2": rel}
        print(f"{nm:>4} {l1:12.4e} {l2:12.4e} {linf:12.4e} {rel:10.2e}", file=out)
    if ncol == 13:
        print("-" * 56, file=out)
        print(f"# divB control (col 12): a L1={np.mean(np.abs(a[:, 11])):.3e} Linf={np.max(np.abs(a[:, 11])):.3e}"
              f"  b L1={np.mean(np.abs(b[:, 11])):.3e} Linf={np.max(np.abs(b[:, 11])):.3e}", file=out)
    return res


def run_case(n, ny, t_end, precision, exact, problem, domain, bc, params):
    with Solver(nx=n, ny=ny, precision=precision, exact=exact, domain=domain, bc=bc) as s:
        s.init_problem(problem, params)
        t0 = time.perf_counter()
        st = s.advance(t_end=t_end)
        wall = time.perf_counter() - t0
        U = s.get_state(LAYOUT_INTERIOR).astype(np.float64)
    return U, st, wall


ALL_RUNS = (("fp64", "fp64", False), ("fp64_exact", "fp64", True), ("fp32", "fp32", False),
            ("mixed", "mixed", False))


def run_study(n, t_end, problem_name, ny=None, runs_wanted=None):
    if problem_name == "kh_reflect":
        problem, domain, bc, params = PROBLEM_KH_REFLECT, (0.0, 1.0, -1.0, 1.0), (0, 0, 1, 1), [0.05, 0.1]
        ny = ny or 2 * n
    else:
        problem, domain, bc, params = PROBLEM_ORSZAG_TANG, (0.0, 1.0, 0.0, 1.0), (0, 0, 0, 0), None
        ny = ny or n
    runs = {}
    states = {}
    for tag, prec, exact in ALL_RUNS:
        if runs_wanted is not None and tag != "fp64" and tag not in runs_wanted:
            continue
        U, st, wall = run_case(n, ny, t_end, prec, exact, problem, domain, bc, params)
        states[tag] = U
        runs[tag] = {"steps": st.steps, "t": st.t, "device_s": st.device_ms / 1e3, "wall_s": wall,
                     "zone_cycles_per_s": n * ny * st.steps / (st.device_ms / 1e3),
                     "hlld_fallbacks": st.degenerate + st.nonphysical}
    ref = states["fp64"]
    prims_ref = conserved_to_dat_columns(ref)
    for tag in [t for t in ("fp64_exact", "fp32", "mixed") if t in states]:
        runs[tag]["relL2_conserved_vs_fp64"] = dict(zip(CONS_NAMES, map(float, relative_l2(ref, states[tag]))))
        runs[tag]["relL2_dat_vs_fp64"] = dict(zip(DAT_NAMES, map(float, relative_l2(
            prims_ref, conserved_to_dat_columns(states[tag])))))
    return {"problem": problem_name, "nx": n, "ny": ny, "t_end": t_end, "runs": runs}


def conv_bench(batch, n, reps=20, seed=7):
    """One GELU 3x3 layer (32 -> 32) over batch x n x n periodic images."""
    import ctypes

    import torch

    from . import CONV_GELU, OK, load, strerror

    g = torch.Generator(device="cpu").manual_seed(seed)
    cin = cout = 32
    x = torch.randn((batch, n, n, cin), generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn((cout, 9, cin), generator=g) * 0.1).to(torch.bfloat16).cuda()
    b = torch.zeros((cout,), dtype=torch.float32, device="cuda")
    z = torch.empty((batch, n, n, cout), dtype=torch.bfloat16, device="cuda")
    a = torch.empty_like(z)
    L = load()

    def call():
        rc = L.pmhd_conv3x3(CONV_GELU, x.data_ptr(), batch, n, n, cin, w.data_ptr(),
                            ctypes.cast(b.data_ptr(), ctypes.POINTER(ctypes.c_float)), cout, None, z.data_ptr(),
                            a.data_ptr(), None)
        if rc != OK:
            raise RuntimeError(strerror(rc))

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        call()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e3)
    us = float(np.median(times))
    pixels = batch * n * n
    flops = 2.0 * 9 * cin * cout * pixels
    nbytes = pixels * (cin + 2 * cout) * 2
    return {"layer": "3x3 conv 32->32 + GELU, bf16 in/out, fp32 accumulation", "batch": batch, "n": n,
            "us_per_call_median": us, "tflops": flops / (us * 1e-6) / 1e12, "hbm_gbs": nbytes / (us * 1e-6) / 1e9,
            "flop_per_call": flops, "algorithmic_bytes_per_call": nbytes, "reps": reps}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m pmhd.study")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("compare")
    c.add_argument("a")
    c.add_argument("b")
    r = sub.add_parser("run")
    r.add_argument("--n", type=int, default=512)
    r.add_argument("--ny", type=int, default=None)
    r.add_argument("--t-end", type=float, default=0.5)
    r.add_argument("--problem", choices=["ot", "kh_reflect"], default="ot")
    r.add_argument("--runs", default=None, help="comma list of fp64_exact, fp32, mixed (fp64 always runs)")
    v = sub.add_parser("conv")
    v.add_argument("--batch", type=int, default=8)
    v.add_argument("--n", type=int, default=512)
    v.add_argument("--reps", type=int, default=20)
    args = ap.parse_args(argv)
    if args.cmd == "compare":
        compare_dat(args.a, args.b)
    elif args.cmd == "conv":
        print(json.dumps(conv_bench(args.batch, args.n, args.reps)))
    else:
        wanted = None if args.runs is None else set(args.runs.split(","))
        print(json.dumps(run_study(args.n, args.t_end, args.problem, args.ny, wanted)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
