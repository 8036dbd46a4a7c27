"""GPU checks of the Euler sibling (pmhd_euler2d_*, pmhd_euler1d_run).

Exact build: every golden run of the reference's 1D and 2D programs
(tests/golden/euler_runs.json), the shock-bubble program at its own 500 x 197
grid included, is reproduced bit for bit (md5 of the .dat the reference
would write) and so is the oracle on rectangular grids with partial tiles
and on step-limited, resumed runs.  Fast build: within rounding-level
tolerances of the oracle.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import euler_lib as EL

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "euler_runs.json")))


@pytest.mark.parametrize("run", GOLD["runs2d"], ids=lambda r: f"{r['n']}-cfg{r['config']}-{r['solver']}-{r['precision']}")
def test_2d_exact_reproduces_the_reference(pmhd_lib, run):
    with pmhd_lib.Euler2D(run["n"], config=run["config"], solver=run["solver"], precision=run["precision"],
                          exact=True) as e:
        st = e.advance()
        assert st.steps == run["steps"]
        assert EL.dat_md5_2d(e.prims(), run["precision"]) == run["md5"]


@pytest.mark.parametrize("run", GOLD["runs1d"], ids=lambda r: f"toro{r['test']}-{r['solver']}-{r['precision']}")
def test_1d_exact_reproduces_the_reference(pmhd_lib, run):
    st, out = pmhd_lib.euler1d(run["n"], run["test"], run["solver"], run["precision"], exact=True)
    assert st.steps == run["steps"]
    assert EL.dat_md5_1d(out, run["precision"]) == run["md5"]


@pytest.mark.parametrize("shape", [(100, 70), (33, 47), (17, 129)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_2d_exact_rectangular_grids_match_the_oracle(oracle, pmhd_lib, shape, prec):
    nx, ny = shape
    steps, t, ref = EL.riemann2d(nx, 6, "hllc", prec, ny=ny)
    with pmhd_lib.Euler2D(nx, ny, config=6, precision=prec, exact=True) as e:
        st = e.advance()
        assert st.steps == steps
        np.testing.assert_array_equal(e.prims(), ref)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_2d_exact_large_grid_matches_the_oracle(oracle, pmhd_lib, prec):
    """640 x 480: enough tiles for the binary64 kernel's 32 x 16 tile shape
    (smaller grids take 32 x 12 tiles); 20 steps, both step orders."""
    steps, t, ref = EL.riemann2d(640, 6, "hllc", prec, ny=480, max_steps=20)
    with pmhd_lib.Euler2D(640, 480, config=6, precision=prec, exact=True) as e:
        assert e.advance(max_steps=20).steps == steps == 20
        np.testing.assert_array_equal(e.prims(), ref)


def test_2d_step_limited_runs_resume_exactly(oracle, pmhd_lib):
    steps, t, ref = EL.riemann2d(80, 12, "hllc", "fp64")
    _, _, ref7 = EL.riemann2d(80, 12, "hllc", "fp64", max_steps=7)
    with pmhd_lib.Euler2D(80, config=12, exact=True) as e:
        assert e.advance(max_steps=7).steps == 7
        np.testing.assert_array_equal(e.prims(), ref7)
        assert e.advance().steps == steps
        np.testing.assert_array_equal(e.prims(), ref)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
@pytest.mark.parametrize("config", [3, 6, 12])
def test_2d_fast_build_close_to_the_oracle(oracle, pmhd_lib, prec, tol, config):
    _, _, ref = EL.riemann2d(128, config, "hllc", prec)
    with pmhd_lib.Euler2D(128, config=config, precision=prec, exact=False) as e:
        e.advance()
        got = e.prims().astype(np.float64)
    rel = pmhd_lib.relative_l2(ref.astype(np.float64), got)
    assert np.all(rel < tol), rel


@pytest.mark.parametrize("test", [1, 2, 3, 4, 5])
def test_1d_fast_build_close_to_the_oracle(oracle, pmhd_lib, test):
    _, _, ref = EL.riemann1d(400, test, "hllc", "fp64")
    st, out = pmhd_lib.euler1d(400, test, "hllc", "fp64", exact=False)
    rel = pmhd_lib.relative_l2(ref, out)
    assert np.all(rel < 1e-10), rel


@pytest.mark.parametrize("run", GOLD["shock_bubble"], ids=lambda r: r["precision"])
def test_shock_bubble_exact_reproduces_the_reference(pmhd_lib, tmp_path, run):
    """src/euler/euler2d_cpu.cpp, 500 x 197 to t = 0.0011741 s: steps, final
    time, and the data lines of the .dat file written by Euler2D.write_dat
    (and of the oracle-side formatter) equal the reference program's."""
    prec = run["precision"]
    T = np.float64 if prec == "fp64" else np.float32
    with pmhd_lib.Euler2D(config="shock_bubble", precision=prec, exact=True) as e:
        st = e.advance()
        assert (e.nx, e.ny) == (run["nx"], run["ny"])
        assert st.steps == run["steps"]
        assert T(st.t) == T(run["t"])
        path = e.write_dat(str(tmp_path / "gpu_shock_bubble.dat"))
        prims = e.prims()
    h = hashlib.md5()
    with open(path, "rb") as f:
        header = [next(f) for _ in range(3)]
        for line in f:
            h.update(line)
    assert header[1] == b"# Steps = %d\n" % run["steps"]
    assert h.hexdigest() == run["md5_data"]
    assert EL.dat_md5_shock_bubble(prims, prec) == run["md5_data"]


@pytest.mark.parametrize("shape", [(120, 50), (77, 33)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_shock_bubble_exact_other_grids_match_the_oracle(oracle, pmhd_lib, shape, prec):
    nx, ny = shape
    steps, t, ref = EL.shock_bubble(nx, ny, "hllc", prec)
    with pmhd_lib.Euler2D(nx, ny, config="shock_bubble", precision=prec, exact=True) as e:
        st = e.advance()
        assert st.steps == steps
        np.testing.assert_array_equal(e.prims(), ref)


def test_shock_bubble_step_limited_runs_resume_exactly(oracle, pmhd_lib):
    steps, t, ref = EL.shock_bubble(100, 40, "hllc", "fp32")
    _, _, ref9 = EL.shock_bubble(100, 40, "hllc", "fp32", max_steps=9)
    with pmhd_lib.Euler2D(100, 40, config="shock_bubble", precision="fp32", exact=True) as e:
        assert e.advance(max_steps=9).steps == 9
        np.testing.assert_array_equal(e.prims(), ref9)
        assert e.advance().steps == steps
        np.testing.assert_array_equal(e.prims(), ref)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
def test_shock_bubble_fast_build_close_to_the_oracle(oracle, pmhd_lib, prec, tol):
    steps, _, ref = EL.shock_bubble(200, 79, "hllc", prec)
    with pmhd_lib.Euler2D(200, 79, config="shock_bubble", precision=prec, exact=False) as e:
        st = e.advance()
        got = e.prims().astype(np.float64)
    assert abs(st.steps - steps) <= 1
    rel = pmhd_lib.relative_l2(ref.astype(np.float64), got)
    print("shock-bubble fast", prec, rel)
    assert np.all(rel < tol), rel
