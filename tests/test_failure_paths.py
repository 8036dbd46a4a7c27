"""Failure paths of the single-grid solver on the GPU, made on the host (no
GPU fault is ever provoked):

  * a non-physical state poked into an Orszag-Tang state on the host and
    uploaded through pmhd_set_state (negative pressure in one cell; NaN
    momentum in another): the exact kernels must stop with the reference's
    status (3 = a stage-1 state, 4 = a stage-2 state; src/mhd/
    mhd2d_glm_gpu.cu:507-531) at the same step and the same first bad cell
    (lowest j * nx + i, the reference's atomicMin, :289-321) as the CPU
    oracle, for every precision policy;
  * the bounded wait of the stage kernel's input load: a test hook
    (PMHD_TEST_STALL_POLLS) makes the first wait of every CTA run out with
    no load issued, so nothing is in flight when the CTAs leave; the advance
    must return PMHD_ERR_TIMEOUT and a fresh handle must then run normally
    (the context stays usable).
"""
import os

import numpy as np
import pytest

from test_gpu_parity import gpu_run, oracle_run

pytestmark = pytest.mark.gpu

NX, NY = 48, 40


def _poked(oracle, prec, kind):
    U = oracle.init_ref_problem("f32" if prec == "fp32" else "f64", 0, NX, NY)
    if kind == "negative_pressure":
        i, j = 17, 23
        c = U[j + 2, i + 2]
        rho, mx, my, mz, E, bx, by, bz = c[:8]
        kinetic = 0.5 * (mx * mx + my * my + mz * mz) / rho
        magnetic = 0.5 * (bx * bx + by * by + bz * bz)
        c[4] = kinetic + magnetic - 0.3 * (E - kinetic - magnetic)  # p < 0
    else:
        i, j = 30, 11
        U[j + 2, i + 2, 1] = np.nan
    return U


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("kind", ["negative_pressure", "nan_momentum"])
def test_poked_state_stops_like_the_oracle(pmhd_lib, oracle, prec, kind):
    U0 = _poked(oracle, prec, kind)
    with pmhd_lib.Solver(nx=NX, ny=NY, precision=prec, exact=True) as s:
        s.set_state(U0, layout=pmhd_lib.LAYOUT_GHOSTED)
        st = s.advance(t_end=0.1, check=False)
    Uo, so = oracle_run(oracle, prec, NX, NY, 0.1, U0=U0)
    assert so.status in (3, 4), so.status
    assert st.status == so.status
    assert (st.bad_i, st.bad_j) == (so.bad_i, so.bad_j)
    assert st.bad_step == so.steps  # the step the failure happened in
    assert st.steps == so.steps


def test_cli_failure_matches_the_reference_failure_report(pmhd_lib, tmp_path):
    """The drop-in program stops where the reference CPU program stops, with
    its message and exit code (tests/golden/runs_large.json, written by the
    reference program)."""
    import json
    import subprocess

    here = os.path.dirname(os.path.abspath(__file__))
    gold = json.load(open(os.path.join(here, "golden", "runs_large.json")))["failures"]
    cli = os.path.join(os.path.dirname(here), "precision-study_b200", "bin", "mhd2d_glm_gpu")
    for rec in gold:
        prog = cli + "_" + rec["precision"]
        args = [str(a) for a in rec["args"]]
        env = dict(os.environ, PMHD_EXACT="1", OUTDIR=str(tmp_path))
        r = subprocess.run([prog] + args, capture_output=True, text=True, env=env, timeout=120)
        assert r.returncode == rec["exit"], (r.returncode, r.stderr)
        assert rec["message"] in r.stderr, (rec["message"], r.stderr)


def test_bounded_wait_expiry_returns_timeout_and_context_survives(pmhd_lib, oracle, monkeypatch):
    monkeypatch.setenv("PMHD_TEST_STALL_POLLS", "1000")
    with pmhd_lib.Solver(nx=64, ny=64, precision="mixed", exact=True) as s:
        s.init_problem(0)
        st = s.advance(t_end=0.05, check=False)
        assert st.status == pmhd_lib.ERR_TIMEOUT
        assert st.steps == 0
    monkeypatch.delenv("PMHD_TEST_STALL_POLLS")
    # A fresh handle in the same process and context runs normally.
    Ug, sg = gpu_run(pmhd_lib, "mixed", 40, 24, 0.06)
    Uo, so = oracle_run(oracle, "mixed", 40, 24, 0.06)
    assert sg.status == 0 and sg.steps == so.steps > 0
    np.testing.assert_array_equal(Ug, Uo)
