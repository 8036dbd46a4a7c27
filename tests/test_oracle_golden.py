"""CPU tests: the oracle and the host-side point interface against golden
fixtures produced by the reference itself (tests/golden/make_golden.py).

Bar: bit-identical outputs and status codes.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")

OPS = {"cons_to_prim": 0, "prim_to_cons": 1, "fast_x": 2, "fast_y": 3, "hll_x": 4, "hll_y": 5,
       "hlld_x": 6, "hlld_y": 7, "glm_hlld_x": 8, "glm_hlld_y": 9, "glm_hll_x": 10, "glm_hll_y": 11,
       "minmod": 12, "positive": 13}
FIXTURES = ["point_fp64", "point_fp32", "point_gamma2_fp64"]


def load_fixture(name):
    d = np.load(os.path.join(GOLD, name + ".npz"))
    return {k: d[k] for k in d.files}


def oracle_eval(oracle, prec, op, x, gamma, tol):
    """Evaluate one golden record with the oracle's exported point functions."""
    L = oracle.lib()
    dt = np.float32 if prec == "f32" else np.float64
    ct = ctypes.c_float if prec == "f32" else ctypes.c_double
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ct))
    a = np.ascontiguousarray(x[:9], dtype=dt)
    b = np.ascontiguousarray(x[9:18], dtype=dt)
    ch = float(x[18])
    out = np.zeros(9, dtype=dt)
    st = 0
    sfx = "_" + prec
    if op == 0:
        getattr(L, "or_point_cons_to_prim" + sfx)(P(a), P(out), gamma)
    elif op == 1:
        getattr(L, "or_point_prim_to_cons" + sfx)(P(a), P(out), gamma)
    elif op in (2, 3):
        out[0] = getattr(L, "or_point_fast_speed" + sfx)(P(a), op - 2, gamma)
    elif op in (4, 5):
        getattr(L, "or_point_hll" + sfx)(P(a), P(b), P(out), op - 4, gamma)
    elif op in (6, 7):
        st = getattr(L, "or_point_hlld" + sfx)(P(a), P(b), P(out), op - 6, gamma, tol)
    elif op in (8, 9, 10, 11):
        hlld = 1 if op in (8, 9) else 0
        st = getattr(L, "or_point_glm_flux" + sfx)(P(a), P(b), ch, hlld, (op - 8) % 2, P(out), gamma, tol)
    elif op == 12:
        out[0] = getattr(L, "or_point_minmod" + sfx)(a[0], b[0])
    elif op == 13:
        st = getattr(L, "or_point_positive" + sfx)(P(a), gamma)
    return st, out


def assert_bitwise(got, want, what):
    g = np.asarray(got)
    w = np.asarray(want)
    same = (g.view(np.uint32 if g.dtype == np.float32 else np.uint64) ==
            w.view(np.uint32 if w.dtype == np.float32 else np.uint64))
    # NaN payload/sign may differ between compilers; NaN-ness must not.
    nan_ok = np.isnan(g) & np.isnan(w)
    assert np.all(same | nan_ok), f"{what}: {g} != {w}"


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_point_functions_match_reference_headers(oracle, name):
    fx = load_fixture(name)
    prec = "f32" if "fp32" in name else "f64"
    gamma, tol = float(fx["gamma"]), float(fx["tol"])
    nops = 0
    for i in range(len(fx["op"])):
        op = int(fx["op"][i])
        st, out = oracle_eval(oracle, prec, op, fx["inp"][i], gamma, tol)
        assert st == fx["status"][i], (name, i, op, st, fx["status"][i])
        assert_bitwise(out, fx["out"][i], f"{name} record {i} op {op}")
        nops += 1
    assert nops > 2000


def test_fixtures_exercise_fallbacks():
    """The golden set must contain both HLLD fallback reasons and clean cases."""
    fx = load_fixture("point_fp64")
    st = fx["status"][np.isin(fx["op"], [6, 7, 8, 9])]
    assert (st == 0).sum() > 100 and (st == 1).sum() > 10 and (st == 2).sum() > 5


@pytest.fixture(scope="module")
def compat_harness(tmp_path_factory):
    """The reference's own point harness compiled against this project's
    drop-in header (include/pmhd/compat) instead of the reference headers."""
    d = tmp_path_factory.mktemp("compat")
    out = {}
    src = os.path.join(ROOT, "oracle", "ref_point_harness.cpp")
    inc = os.path.join(ROOT, "include", "pmhd", "compat")
    for name, extra in (("point_fp64", ["-DMHD_GAMMA_VALUE=(5.0/3.0)"]),
                        ("point_fp32", ["-DMHD_GAMMA_VALUE=(5.0/3.0)", "-DUSE_FLOAT"]),
                        ("point_gamma2_fp64", ["-DMHD_GAMMA_VALUE=2.0"])):
        exe = str(d / name)
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", inc,
                        "-DMHD_HLLD_TOLERANCE_VALUE=1.0e-4"] + extra + [src, "-o", exe], check=True)
        out[name] = exe
    return out


@pytest.mark.parametrize("name", FIXTURES)
def test_compat_header_matches_reference_headers(compat_harness, name):
    """pmhd/point.hpp (through the reference-named compat API) gives the same
    bits and status codes as the reference headers for every golden record."""
    sys.path.insert(0, GOLD)
    import make_golden
    fx = load_fixture(name)
    dt = np.float32 if "fp32" in name else np.float64
    recs = [(int(o), x) for o, x in zip(fx["op"], fx["inp"])]
    status, res = make_golden.run_harness(compat_harness[name], recs, dt)
    np.testing.assert_array_equal(status, fx["status"])
    for i in range(len(recs)):
        assert_bitwise(res[i], fx["out"][i], f"{name} record {i}")


RUNS = json.load(open(os.path.join(GOLD, "runs.json")))["runs"]


@pytest.mark.parametrize("run", RUNS, ids=lambda r: "{precision}-{nx}x{ny}-{order}-{solver}".format(**r))
def test_oracle_runs_match_reference_solver_output(oracle, run, tmp_path):
    prec = "f32" if run["precision"] == "fp32" else "f64"
    cfg = oracle.make_config(run["nx"], run["ny"], run["t_end"], cfl=run["cfl"], alpha=run["alpha"],
                             muscl=run["order"] == "muscl", hlld=run["solver"] == "hlld")
    U = oracle.init_ref_problem(prec, 0, run["nx"], run["ny"])
    st = oracle.run(prec, cfg, U)
    assert st.status == 0 and st.steps == run["steps"]
    assert (st.degenerate, st.nonphysical) == (run["degenerate"], run["nonphysical"])
    assert (st.x_evals, st.y_evals) == (run["x_evals"], run["y_evals"])
    assert float("%.6g" % st.ch_last) == run["ch_last_printed"]
    assert oracle.dat_lines_md5(prec, cfg, U, str(tmp_path / "o.dat")) == run["md5"]


def test_planted_mistake_is_detected(oracle, tmp_path):
    """A perturbed oracle run (HLLD tolerance 1e-6 instead of 1e-4) must not
    reproduce the golden md5, so the md5 comparison above has teeth."""
    run = RUNS[4]
    cfg = oracle.make_config(run["nx"], run["ny"], run["t_end"], tol=1e-6)
    U = oracle.init_ref_problem("f64", 0, run["nx"], run["ny"])
    oracle.run("f64", cfg, U)
    assert oracle.dat_lines_md5("f64", cfg, U, str(tmp_path / "p.dat")) != run["md5"]


@pytest.mark.slow
@pytest.mark.parametrize("prec,steps,deg,nonphys,md5", [
    ("f64", 1936, 13370, 2, "4fe78b53eebc633b94d04b01b37ebbca"),
    ("f32", 1936, 13362, 2, "dfa6392909b0b20979fa4a45b9a1334d"),
])
def test_oracle_ot192_matches_reference_logs(oracle, prec, steps, deg, nonphys, md5, tmp_path):
    """Reference logs logs/mhd/ot_large_eps1e-4_20260715/mhd2d_fp{64,32}_eps1e-4_N192.log
    (steps, fallback counts) and the data-line md5 of the reference output."""
    cfg = oracle.make_config(192, 192, 0.5)
    U = oracle.init_ref_problem(prec, 0, 192, 192)
    st = oracle.run(prec, cfg, U)
    assert (st.steps, st.degenerate, st.nonphysical) == (steps, deg, nonphys)
    assert oracle.dat_lines_md5(prec, cfg, U, str(tmp_path / "o.dat")) == md5


def test_mixed_oracle_close_to_f64(oracle):
    """The mixed restatement stays within binary32 rounding of binary64 on a
    short run (its own bar is parity with the GPU mixed kernels)."""
    cfg = oracle.make_config(48, 48, 0.05)
    Ua = oracle.init_ref_problem("f64", 0, 48, 48)
    Ub = Ua.copy()
    sa = oracle.run("f64", cfg, Ua)
    sb = oracle.run("mixed", cfg, Ub)
    assert sa.steps == sb.steps
    d = Ua[2:-2, 2:-2, :8] - Ub[2:-2, 2:-2, :8]
    rel = np.sqrt((d ** 2).mean(axis=(0, 1))) / np.maximum(np.sqrt((Ua[2:-2, 2:-2, :8] ** 2).mean(axis=(0, 1))), 1e-30)
    assert np.all(rel[[0, 1, 2, 4, 5, 6]] < 1e-5), rel


LARGE = json.load(open(os.path.join(GOLD, "runs_large.json")))


@pytest.mark.parametrize("fail", LARGE["failures"], ids=lambda r: r["precision"])
def test_oracle_failure_report_matches_reference(oracle, fail):
    """The oracle stops where the reference CPU program stops on a run that
    meets a non-physical stage: same status (exit code), step and first bad
    cell (tests/golden/runs_large.json, written by the reference program)."""
    nx, ny, t_end, cfl, order, solver, alpha = fail["args"]
    prec = "f32" if fail["precision"] == "fp32" else "f64"
    cfg = oracle.make_config(nx, ny, t_end, cfl=cfl, alpha=alpha, muscl=order == "muscl", hlld=solver == "hlld")
    U = oracle.init_ref_problem(prec, 0, nx, ny)
    st = oracle.run(prec, cfg, U)
    assert st.status == fail["exit"]
    assert (st.steps, st.bad_i, st.bad_j) == (fail["step"], fail["i"], fail["j"])


@pytest.mark.slow
@pytest.mark.parametrize("run", LARGE["runs"], ids=lambda r: r["precision"])
def test_oracle_ot256_matches_reference_output(oracle, run, tmp_path):
    """The plain-method configuration (Orszag-Tang 256^2 to t = 0.5): the
    oracle reproduces the reference program's step count, counters and
    data-line md5 (about ten minutes of CPU)."""
    prec = "f32" if run["precision"] == "fp32" else "f64"
    cfg = oracle.make_config(256, 256, 0.5)
    U = oracle.init_ref_problem(prec, 0, 256, 256)
    st = oracle.run(prec, cfg, U)
    assert (st.steps, st.degenerate, st.nonphysical) == (run["steps"], run["degenerate"], run["nonphysical"])
    assert oracle.dat_lines_md5(prec, cfg, U, str(tmp_path / "o.dat")) == run["md5"]
