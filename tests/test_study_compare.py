"""`python -m pmhd.study compare A.dat B.dat` (the reference's
analysis/mhd/compare_precision.py table) on .dat files written in the
reference format by the oracle: layout detection, and relL2 = RMS(a - b) /
RMS(a) per column, zero for identical files."""
import io
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "precision-study_b200"))


def _write(oracle, path, U, nx, ny):
    oracle.dat_lines_md5("f64", oracle.make_config(nx, ny, 0.0), U, str(path))


def test_compare_identical_and_perturbed_files(oracle, tmp_path):
    from pmhd import study
    nx, ny = 16, 12
    U = oracle.init_ref_problem("f64", 0, nx, ny)
    a, b, c = tmp_path / "a.dat", tmp_path / "b.dat", tmp_path / "c.dat"
    _write(oracle, a, U, nx, ny)
    _write(oracle, b, U, nx, ny)
    V = U.copy()
    V[..., 0] *= 1.0 + 1e-3  # density scaled: rho relL2 = 1e-3 (to the file's printed digits)
    _write(oracle, c, V, nx, ny)
    out = io.StringIO()
    same = study.compare_dat(str(a), str(b), out=out)
    assert "2D OT-GLM" in out.getvalue() and f"N = {nx * ny}" in out.getvalue()
    assert all(v["relL2"] == 0.0 for v in same.values())
    diff = study.compare_dat(str(a), str(c), out=io.StringIO())
    assert diff["rho"]["relL2"] == pytest.approx(1e-3, rel=1e-6)
    # the velocities are momenta over density: they move by the same factor
    assert diff["vx"]["relL2"] == pytest.approx(1e-3 / (1.0 + 1e-3), rel=1e-6)
    assert diff["Bx"]["relL2"] == 0.0


def test_compare_rejects_mismatched_shapes(oracle, tmp_path):
    from pmhd import study
    U1 = oracle.init_ref_problem("f64", 0, 8, 8)
    U2 = oracle.init_ref_problem("f64", 0, 8, 10)
    a, b = tmp_path / "a.dat", tmp_path / "b.dat"
    _write(oracle, a, U1, 8, 8)
    _write(oracle, b, U2, 8, 10)
    with pytest.raises(SystemExit):
        study.compare_dat(str(a), str(b), out=io.StringIO())
