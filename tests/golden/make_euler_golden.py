#!/usr/bin/env python3
"""Generates tests/golden/euler_runs.json from the reference's own Euler
programs (src/euler/riemann1d_cpu.cpp, src/euler/riemann2d_cpu.cpp,
src/euler/euler2d_cpu.cpp), built by `make -C oracle ref` into oracle/_ref/
(fp64, fp32 = -DUSE_FLOAT, 2D HLL = -DUSE_HLL).  For each run it records the
step count and the md5 of the .dat file the program writes (one line per
cell: x y rho u v p in 2D, x rho u p in 1D; scientific with max_digits10
digits; for the shock-bubble program, whose grid and end time are
compile-time constants, the md5 of its data lines -- those not starting with
'#' -- and the final time from its '# Time' line), so tests can check the
oracle and the GPU kernels bit for bit without the reference present.

Run from the repository root:  python tests/golden/make_euler_golden.py
"""
import hashlib
import json
import os
import re
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "euler_runs.json")

RUNS_2D = [(64, 3, "hllc", "fp64"), (64, 6, "hllc", "fp64"), (64, 12, "hllc", "fp64"), (100, 3, "hllc", "fp64"),
           (64, 3, "hllc", "fp32"), (64, 6, "hllc", "fp32"), (64, 12, "hllc", "fp32"), (64, 6, "hll", "fp64"),
           (64, 3, "hll", "fp64")]
RUNS_1D = [(200, t, s, p) for t in range(1, 6) for s, p in (("hllc", "fp64"), ("hllc", "fp32"), ("hll", "fp64"))]


def run(cmd, outdir):
    env = dict(os.environ, OUTDIR=outdir)
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, check=True)
    steps = int(re.search(r"Done\. Steps: (\d+)", r.stdout).group(1))
    path = re.search(r"Saved: (\S+)", r.stdout).group(1)
    with open(path, "rb") as f:
        return steps, hashlib.md5(f.read()).hexdigest()


def run_shock_bubble(exe, outdir):
    env = dict(os.environ, OUTDIR=outdir)
    r = subprocess.run([exe], env=env, capture_output=True, text=True, check=True)
    steps = int(re.search(r"Done\. Steps: (\d+)", r.stdout).group(1))
    h = hashlib.md5()
    t = None
    with open(os.path.join(outdir, "cpu_shock_bubble.dat"), "rb") as f:
        for line in f:
            if line.startswith(b"# Time = "):
                t = float(line.split(b"=")[1])
            if not line.startswith(b"#"):
                h.update(line)
    return steps, t, h.hexdigest()


def main():
    out = {"generator": "tests/golden/make_euler_golden.py",
           "reference": "src/euler/{riemann1d,riemann2d,euler2d}_cpu.cpp built -O2 -ffp-contract=off (oracle/Makefile)",
           "runs2d": [], "runs1d": [], "shock_bubble": []}
    with tempfile.TemporaryDirectory() as tmp:
        for prec in ("fp64", "fp32"):
            steps, t, md5 = run_shock_bubble(os.path.join(REF_DIR, "euler2d_cpu_" + prec), tmp)
            out["shock_bubble"].append({"nx": 500, "ny": 197, "solver": "hllc", "precision": prec, "steps": steps,
                                        "t": t, "md5_data": md5})
        for n, cfg, solver, prec in RUNS_2D:
            exe = os.path.join(REF_DIR, "riemann2d_cpu_" + ("hll_" if solver == "hll" else "") + prec)
            steps, md5 = run([exe, str(n), str(cfg)], tmp)
            out["runs2d"].append({"n": n, "config": cfg, "solver": solver, "precision": prec, "steps": steps,
                                  "md5": md5})
        for n, test, solver, prec in RUNS_1D:
            exe = os.path.join(REF_DIR, "riemann1d_cpu_" + prec)
            steps, md5 = run([exe, str(n), str(test), solver], tmp)
            out["runs1d"].append({"n": n, "test": test, "solver": solver, "precision": prec, "steps": steps,
                                  "md5": md5})
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
