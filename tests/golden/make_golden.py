#!/usr/bin/env python3
"""Generates the golden fixtures in tests/golden/ from the reference itself.

Needs the reference's CPU programs built from its source tree by
`make -C oracle ref REF=<tree>` (or with PMHD_REF=<tree> in the environment)
into oracle/_ref/.  Writes:

  point_fp64.npz, point_fp32.npz, point_gamma2_fp64.npz
      inputs and outputs of the reference's header-only point functions
      (include/mhd/mhd_common.hpp, include/mhd/mhd_glm_common.hpp) run
      through oracle/ref_point_harness.cpp: cons<->prim, fast speeds, HLL,
      HLLD (with status), the GLM fluxes, minmod and the positivity test, on
      seeded random states plus degenerate ones (B_n ~ 0, equal states,
      near vacuum, strong field, non-physical).
  runs.json
      data-line md5 (the reference's own regression gate: md5 of the
      non-'#' lines of the .dat output) and summary numbers of the reference
      CPU solver src/mhd/mhd2d_glm_cpu.cpp on small Orszag-Tang grids, fp64
      and fp32, all order/solver combinations.
  runs_large.json  (--large; about five minutes of CPU per run)
      the same for the plain-method configuration Orszag-Tang 256^2 to
      t = 0.5 (MUSCL, HLLD, CFL 0.25, alpha 0.18), fp64 and fp32, and the
      reference's failure report (exit code, step, cell) of a run that meets
      a non-physical stage.

Run from the repository root:  python tests/golden/make_golden.py [--large]
"""
import hashlib
import json
import os
import re
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203

OPS = {"cons_to_prim": 0, "prim_to_cons": 1, "fast_x": 2, "fast_y": 3, "hll_x": 4, "hll_y": 5,
       "hlld_x": 6, "hlld_y": 7, "glm_hlld_x": 8, "glm_hlld_y": 9, "glm_hll_x": 10, "glm_hll_y": 11,
       "minmod": 12, "positive": 13}


def prim_to_cons(W, gamma):
    rho, vx, vy, vz, p, bx, by, bz = W[:8]
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz)
    return np.array([rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, W[8] if len(W) > 8 else 0.0])


def random_prims(rng, n):
    W = np.empty((n, 9))
    W[:, 0] = rng.uniform(0.05, 3.0, n)
    W[:, 1:4] = rng.uniform(-2.0, 2.0, (n, 3))
    W[:, 4] = rng.uniform(0.01, 3.0, n)
    W[:, 5:8] = rng.uniform(-2.0, 2.0, (n, 3))
    W[:, 8] = rng.uniform(-0.1, 0.1, n)
    return W


def special_pairs(rng, gamma):
    """Left/right conserved states that exercise the guards."""
    pairs = []
    for _ in range(40):
        W = random_prims(rng, 2)
        W[:, 5] = rng.choice([0.0, 1e-9, -1e-9, 1e-5, 0.5])  # normal field ~ 0
        pairs.append(W)
    for _ in range(20):
        W = random_prims(rng, 1)
        pairs.append(np.vstack([W, W]))  # equal states
    for _ in range(20):
        W = random_prims(rng, 2)
        W[:, 0] = rng.choice([1e-11, 1e-6, 1e-3], 2)  # near vacuum
        W[:, 4] = rng.choice([1e-11, 1e-6, 1e-3], 2)
        pairs.append(W)
    for _ in range(20):
        W = random_prims(rng, 2)
        W[:, 5:8] *= 50.0  # strongly magnetised
        pairs.append(W)
    for _ in range(20):
        W = random_prims(rng, 2)
        W[:, 1] = rng.uniform(-20, 20, 2)  # supersonic left/right
        pairs.append(W)
    out = []
    for W in pairs:
        out.append((prim_to_cons(W[0], gamma), prim_to_cons(W[1], gamma)))
    for _ in range(20):  # non-physical: negative pressure or density
        a, b = random_prims(rng, 2)
        ua, ub = prim_to_cons(a, gamma), prim_to_cons(b, gamma)
        ua[4] -= rng.uniform(0.5, 5.0) * abs(ua[4])
        if rng.random() < 0.5:
            ub[0] = -abs(ub[0])
        out.append((ua, ub))
    return out


def build_records(gamma, rng):
    recs = []  # (op, in19)
    W = random_prims(rng, 200)
    pairs = [(prim_to_cons(W[2 * i], gamma), prim_to_cons(W[2 * i + 1], gamma)) for i in range(100)]
    pairs += special_pairs(rng, gamma)
    for ua, ub in pairs:
        ch = rng.choice([0.0, 1e-13, 0.7, 2.5])
        for name in ("hll_x", "hll_y", "hlld_x", "hlld_y", "glm_hlld_x", "glm_hlld_y", "glm_hll_x",
                     "glm_hll_y"):
            recs.append((OPS[name], np.concatenate([ua, ub, [ch]])))
        for name in ("cons_to_prim", "positive"):
            recs.append((OPS[name], np.concatenate([ua, ub, [0.0]])))
    for w in random_prims(rng, 100):
        recs.append((OPS["prim_to_cons"], np.concatenate([w, np.zeros(10)])))
        for name in ("fast_x", "fast_y"):
            recs.append((OPS[name], np.concatenate([w, np.zeros(10)])))
    vals = rng.normal(size=(200, 2)) * rng.choice([1e-8, 1.0, 1e3], (200, 1))
    vals[:20, 1] = 0.0
    vals[20:40, 1] = -vals[20:40, 0]
    vals[40:50, 1] = vals[40:50, 0]
    for a, b in vals:
        x = np.zeros(19)
        x[0], x[9] = a, b
        recs.append((OPS["minmod"], x))
    return recs


def run_harness(binary, recs, dtype):
    fmt = "f" if dtype == np.float32 else "d"
    size = 4 if dtype == np.float32 else 8
    buf = bytearray(struct.pack("i", len(recs)))
    for op, x in recs:
        buf += struct.pack("i", op) + np.asarray(x, dtype=dtype).tobytes()
    out = subprocess.run([binary], input=bytes(buf), capture_output=True, check=True).stdout
    rec = 4 + 9 * size
    assert len(out) == rec * len(recs)
    status = np.empty(len(recs), dtype=np.int32)
    res = np.empty((len(recs), 9), dtype=dtype)
    for i in range(len(recs)):
        status[i] = struct.unpack_from("i", out, i * rec)[0]
        res[i] = np.frombuffer(out, dtype=dtype, count=9, offset=i * rec + 4)
    return status, res


def make_point_fixtures():
    for name, binary, dtype, gamma in (("point_fp64", "ref_point_fp64", np.float64, 5.0 / 3.0),
                                       ("point_fp32", "ref_point_fp32", np.float32, 5.0 / 3.0),
                                       ("point_gamma2_fp64", "ref_point_gamma2_fp64", np.float64, 2.0)):
        rng = np.random.default_rng(SEED)
        recs = build_records(gamma, rng)
        status, res = run_harness(os.path.join(REF_DIR, binary), recs, dtype)
        ops = np.array([r[0] for r in recs], dtype=np.int32)
        ins = np.array([r[1] for r in recs]).astype(dtype)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), op=ops, inp=ins, status=status, out=res,
                            gamma=np.float64(gamma), tol=np.float64(1e-4))
        print(name, len(recs), "records")


def data_md5(path):
    h = hashlib.md5()
    with open(path, "rb") as f:
        for line in f:
            if not line.startswith(b"#"):
                h.update(line)
    return h.hexdigest()


RUNS = [
    # (nx, ny, t_end, cfl, order, solver, alpha)
    (32, 32, 0.1, 0.25, "muscl", "hlld", 0.18),
    (24, 40, 0.15, 0.3, "first", "hll", 0.5),
    (40, 24, 0.12, 0.25, "muscl", "hll", 0.18),
    (32, 32, 0.08, 0.25, "first", "hlld", 0.18),
    (64, 64, 0.2, 0.25, "muscl", "hlld", 0.18),
    (48, 16, 0.1, 0.4, "muscl", "hlld", 1.0),
]


def make_run_fixtures():
    out = []
    with tempfile.TemporaryDirectory() as d:
        for prec in ("fp64", "fp32"):
            binary = os.path.join(REF_DIR, f"mhd2d_glm_cpu_{prec}")
            for nx, ny, t_end, cfl, order, solver, alpha in RUNS:
                env = dict(os.environ, OUTDIR=d)
                r = subprocess.run([binary, str(nx), str(ny), repr(t_end), repr(cfl), order, solver, repr(alpha)],
                                   capture_output=True, text=True, env=env, check=True)
                fn = os.path.join(d, f"orszag_tang_glm_{order}_{solver}_{prec}_N{nx}x{ny}.dat")
                steps = int(re.search(r"Steps: (\d+)", r.stdout).group(1))
                ch = float(re.search(r"c_h\(last\) = ([0-9.eE+-]+)", r.stdout).group(1))
                m = re.search(r"degenerate=(\d+), nonphysical=(\d+)", r.stdout)
                ev = re.search(r"HLLD flux evaluations = (\d+) \(x=(\d+), y=(\d+)\)", r.stdout)
                out.append({"precision": prec, "nx": nx, "ny": ny, "t_end": t_end, "cfl": cfl, "order": order,
                            "solver": solver, "alpha": alpha, "steps": steps, "ch_last_printed": ch,
                            "degenerate": int(m.group(1)) if m else 0, "nonphysical": int(m.group(2)) if m else 0,
                            "x_evals": int(ev.group(2)) if ev else 0, "y_evals": int(ev.group(3)) if ev else 0,
                            "md5": data_md5(fn)})
                print(out[-1])
    with open(os.path.join(OUT, "runs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "reference": "src/mhd/mhd2d_glm_cpu.cpp "
                   "built -O2 -DMHD_HLLD_TOLERANCE_VALUE=1.0e-4 (oracle/Makefile)", "runs": out}, f, indent=1)


def _run_summary(stdout, path):
    steps = int(re.search(r"Steps: (\d+)", stdout).group(1))
    m = re.search(r"degenerate=(\d+), nonphysical=(\d+)", stdout)
    ev = re.search(r"HLLD flux evaluations = (\d+) \(x=(\d+), y=(\d+)\)", stdout)
    dv = re.search(r"divB L1 = ([0-9.eE+-]+), divB Linf = ([0-9.eE+-]+), psi Linf = ([0-9.eE+-]+)", stdout)
    return {"steps": steps, "ch_last_printed": float(re.search(r"c_h\(last\) = ([0-9.eE+-]+)", stdout).group(1)),
            "degenerate": int(m.group(1)), "nonphysical": int(m.group(2)),
            "x_evals": int(ev.group(2)), "y_evals": int(ev.group(3)),
            "divb_line": dv.group(0) if dv else None, "md5": data_md5(path)}


# A run that meets a non-physical state: first order, HLLD, CFL 0.95 and
# alpha 0.01 on Orszag-Tang 32^2 (the reference stops in stage 1 of step 15).
FAILING = (32, 32, 0.5, 0.95, "first", "hlld", 0.01)


def make_large_run_fixtures():
    out = {"generator": "tests/golden/make_golden.py --large",
           "reference": "src/mhd/mhd2d_glm_cpu.cpp built -O2 -DMHD_HLLD_TOLERANCE_VALUE=1.0e-4 (oracle/Makefile)",
           "runs": [], "failures": []}
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for prec in ("fp64", "fp32"):
            binary = os.path.join(REF_DIR, f"mhd2d_glm_cpu_{prec}")
            env = dict(os.environ, OUTDIR=os.path.join(d, prec))
            args = [binary, "256", "256", "0.5", "0.25", "muscl", "hlld", "0.18"]
            procs.append((prec, subprocess.Popen(args, stdout=subprocess.PIPE, text=True, env=env)))
        for prec, p in procs:
            stdout, _ = p.communicate()
            assert p.returncode == 0, prec
            fn = os.path.join(d, prec, f"orszag_tang_glm_muscl_hlld_{prec}_N256x256.dat")
            rec = {"precision": prec, "nx": 256, "ny": 256, "t_end": 0.5, "cfl": 0.25, "order": "muscl",
                   "solver": "hlld", "alpha": 0.18}
            rec.update(_run_summary(stdout, fn))
            out["runs"].append(rec)
            print(rec)
        for prec in ("fp64", "fp32"):
            binary = os.path.join(REF_DIR, f"mhd2d_glm_cpu_{prec}")
            nx, ny, t_end, cfl, order, solver, alpha = FAILING
            r = subprocess.run([binary, str(nx), str(ny), repr(t_end), repr(cfl), order, solver, repr(alpha)],
                               capture_output=True, text=True, env=dict(os.environ, OUTDIR=d))
            m = re.search(r"Error: (non-physical RK stage|non-physical state) at step (\d+), cell \((\d+), (\d+)\)",
                          r.stderr)
            rec = {"precision": prec, "args": [nx, ny, t_end, cfl, order, solver, alpha], "exit": r.returncode,
                   "message": m.group(0), "step": int(m.group(2)), "i": int(m.group(3)), "j": int(m.group(4))}
            out["failures"].append(rec)
            print(rec)
    with open(os.path.join(OUT, "runs_large.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if not os.path.exists(os.path.join(REF_DIR, "ref_point_fp64")):
        sys.exit("build the reference programs first: make -C oracle ref")
    if "--large" in sys.argv[1:]:
        make_large_run_fixtures()
    else:
        make_point_fixtures()
        make_run_fixtures()
