"""CPU checks of the Euler sibling's oracle (oracle/euler_oracle.h): bit
for bit against the reference's own 1D / 2D programs (md5 of their .dat
output, tests/golden/euler_runs.json) and, for the Toro tests, the density
errors against the exact Riemann solution that the reference reports
(tests/golden/exact_riemann_norms.json)."""
import json
import os
import sys

import numpy as np
import pytest

import euler_lib as EL

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import exact_riemann  # noqa: E402

GOLD = json.load(open(os.path.join(HERE, "golden", "euler_runs.json")))
NORMS = json.load(open(os.path.join(HERE, "golden", "exact_riemann_norms.json")))


@pytest.mark.parametrize("run", GOLD["runs2d"], ids=lambda r: f"{r['n']}-cfg{r['config']}-{r['solver']}-{r['precision']}")
def test_oracle_2d_reproduces_the_reference_output(oracle, run):
    steps, t, prims = EL.riemann2d(run["n"], run["config"], run["solver"], run["precision"])
    assert steps == run["steps"]
    assert EL.dat_md5_2d(prims, run["precision"]) == run["md5"]


@pytest.mark.parametrize("run", GOLD["runs1d"], ids=lambda r: f"toro{r['test']}-{r['solver']}-{r['precision']}")
def test_oracle_1d_reproduces_the_reference_output(oracle, run):
    steps, t, out = EL.riemann1d(run["n"], run["test"], run["solver"], run["precision"])
    assert steps == run["steps"]
    assert EL.dat_md5_1d(out, run["precision"]) == run["md5"]


@pytest.mark.parametrize("test", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_density_errors_against_the_exact_solution(oracle, test, prec):
    rl, ul, pl, rr, ur, pr, t_end, x0 = NORMS["states"][str(test)]
    _, _, out = EL.riemann1d(200, test, "hllc", prec)
    x = (np.arange(200) + 0.5) / 200
    rho, _, _ = exact_riemann.solution(rl, ul, pl, rr, ur, pr, x0, t_end, x)
    d = np.abs(out[:, 0].astype(np.float64) - rho)
    ref = NORMS["tests"][str(test)]
    for got, want in ((d.mean(), ref["L1"]), (np.sqrt((d * d).mean()), ref["L2"]), (d.max(), ref["Linf"])):
        assert float("%.3e" % got) == want


def test_exact_solver_conserves_the_sod_star_state():
    # Toro (2009) table 4.2, test 1: p* = 0.30313, u* = 0.92745.
    p, u = exact_riemann.star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    assert abs(p - 0.30313) < 5e-6 and abs(u - 0.92745) < 5e-6


def test_oracle_shock_bubble_reproduces_the_reference_output(oracle):
    """The shock-bubble program (src/euler/euler2d_cpu.cpp) at its own grid,
    500 x 197 to t = 0.0011741 s (3459 steps): step count, final time and the
    md5 of the .dat data lines equal the reference program's, binary64 and
    binary32 (whose time control mixes in binary64 constants).  The two runs
    go concurrently (ctypes releases the GIL during the oracle call)."""
    from concurrent.futures import ThreadPoolExecutor

    runs = GOLD["shock_bubble"]
    with ThreadPoolExecutor(len(runs)) as ex:
        results = list(ex.map(lambda r: EL.shock_bubble(r["nx"], r["ny"], r["solver"], r["precision"]), runs))
    for run, (steps, t, prims) in zip(runs, results):
        T = np.float64 if run["precision"] == "fp64" else np.float32
        assert steps == run["steps"], run["precision"]
        assert T(t) == T(run["t"]), run["precision"]
        assert EL.dat_md5_shock_bubble(prims, run["precision"]) == run["md5_data"], run["precision"]
