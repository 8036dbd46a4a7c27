"""CPU tests of the C ABI boundary (include/pmhd.h, libpmhd.so) and the
drop-in CLI's host-side behaviour.  No kernel runs here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HEADER = os.path.join(ROOT, "include", "pmhd.h")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(pmhd_\w+)\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol(pmhd_lib):
    names = declared_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", pmhd_lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (pmhd_\w+)$", out, flags=re.M))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert sorted(pmhd_lib.EXPORTS) == names


def test_config_defaults_are_reference_cli_defaults(pmhd_lib):
    c = pmhd_lib.default_config()
    assert (c.nx, c.ny) == (128, 128)
    assert (c.x_min, c.x_max, c.y_min, c.y_max) == (0.0, 1.0, 0.0, 1.0)
    assert c.gamma == 5.0 / 3.0 and c.hlld_tol == 1e-4 and c.cfl == 0.25 and c.alpha == 0.18
    assert c.order == pmhd_lib.ORDER_MUSCL and c.solver == pmhd_lib.SOLVER_HLLD
    assert c.precision == pmhd_lib.FP64 and list(c.bc) == [0, 0, 0, 0]


@pytest.mark.parametrize("field,value", [("nx", 2), ("ny", 0), ("cfl", 1.0), ("cfl", 0.0), ("alpha", 0.0),
                                         ("gamma", 1.0), ("order", 7), ("solver", 3), ("precision", 5),
                                         ("steps_per_graph", 3)])
def test_create_rejects_bad_config_before_touching_a_device(pmhd_lib, field, value):
    c = pmhd_lib.default_config()
    setattr(c, field, value)
    h = ctypes.c_void_p(1)
    rc = pmhd_lib.load().pmhd_create(ctypes.byref(c), ctypes.byref(h))
    assert rc == pmhd_lib.ERR_ARG and h.value is None


def test_create_rejects_unpaired_periodic_sides(pmhd_lib):
    c = pmhd_lib.default_config()
    c.bc[0] = pmhd_lib.BC_PERIODIC
    c.bc[1] = pmhd_lib.BC_REFLECT
    h = ctypes.c_void_p()
    assert pmhd_lib.load().pmhd_create(ctypes.byref(c), ctypes.byref(h)) == pmhd_lib.ERR_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly(pmhd_lib):
    with pytest.raises(pmhd_lib.PmhdError) as e:
        pmhd_lib.Solver(nx=16, ny=16)
    assert e.value.status == pmhd_lib.ERR_NODEVICE


def test_null_handles_are_rejected(pmhd_lib):
    L = pmhd_lib.load()
    st = pmhd_lib.Stats()
    assert L.pmhd_advance(None, 1.0, -1, ctypes.byref(st)) == pmhd_lib.ERR_ARG
    assert L.pmhd_get_state(None, None, 0) == pmhd_lib.ERR_ARG
    assert L.pmhd_destroy(None) == pmhd_lib.OK
    assert pmhd_lib.strerror(3) == "non-physical RK stage"
    assert pmhd_lib.strerror(4) == "non-physical state"


@pytest.mark.parametrize("prec,oprec,problem", [("fp64", "f64", 0), ("fp32", "f32", 0), ("fp64", "f64", 1),
                                                ("fp32", "f32", 1), ("mixed", "f64", 0)])
def test_host_initial_conditions_match_oracle(pmhd_lib, oracle, prec, oprec, problem):
    """The library's Orszag-Tang and reference-KH states are bit-identical to
    the oracle's restatement of the reference initial conditions."""
    U = pmhd_lib.problem_state(problem, nx=40, ny=24, precision=prec)
    Uo = oracle.init_ref_problem(oprec, problem, 40, 24)
    np.testing.assert_array_equal(U, Uo)


def test_host_problem_variants(pmhd_lib):
    """KH with reflecting walls and the rotated Brio-Wu tube: basic structure."""
    U = pmhd_lib.problem_state(pmhd_lib.PROBLEM_KH_REFLECT, [0.05, 0.1], nx=32, ny=64,
                               domain=(0.0, 1.0, -1.0, 1.0), bc=(0, 0, 1, 1))
    rho = U[2:-2, 2:-2, 0]
    assert np.allclose(rho, 1.0) and np.allclose(U[2:-2, 2:-2, 5], 0.1)
    vx = U[2:-2, 2:-2, 1] / rho
    assert vx[0].mean() < -0.45 and vx[-1].mean() > 0.45
    B = pmhd_lib.problem_state(pmhd_lib.PROBLEM_BRIO_WU_2D, [np.pi / 4], nx=32, ny=32, gamma=2.0,
                               bc=(2, 2, 2, 2))
    bx, by = B[2:-2, 2:-2, 5], B[2:-2, 2:-2, 6]
    bn = (bx + by) / np.sqrt(2.0)  # normal of the 45-degree interface
    assert np.allclose(bn, 0.75)
    assert set(np.round(B[2:-2, 2:-2, 0], 6).ravel()) == {1.0, 0.125}


def test_relative_l2_definition(pmhd_lib):
    a = np.random.default_rng(0).normal(size=(10, 10, 9))
    assert np.all(pmhd_lib.relative_l2(a, a) == 0)
    b = a * (1 + 1e-3)
    np.testing.assert_allclose(pmhd_lib.relative_l2(a, b), 1e-3, rtol=1e-9)


CLI = os.path.join(ROOT, "precision-study_b200", "bin", "mhd2d_glm_gpu")


@pytest.mark.parametrize("args,msg", [(["16", "16", "0.1", "0.25", "weno"], "order must be"),
                                      (["16", "16", "0.1", "0.25", "muscl", "roe"], "solver must be"),
                                      (["16", "16", "0.1", "0.25", "muscl", "hlld", "-1"], "alpha must be"),
                                      (["16", "16", "0.1", "0.25", "muscl", "hlld", "0.18", "sod"],
                                       "problem must be")])
def test_cli_argument_errors_exit_1(pmhd_lib, args, msg):
    r = subprocess.run([CLI] + args, capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_cli_without_device_exits_9(pmhd_lib):
    r = subprocess.run([CLI, "16", "16", "0.01"], capture_output=True, text=True)
    assert r.returncode == 9
    assert "Orszag-Tang" in r.stdout


EULER_CLI = os.path.join(ROOT, "precision-study_b200", "bin", "euler2d_gpu")


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_euler_cli_without_device_exits_1(pmhd_lib):
    """The shock-bubble drop-in prints the reference program's header lines
    (euler2d_cuda.cu:290-296, :226-243, with its logged shock states) and,
    without a B200, exits with EXIT_FAILURE as the reference's CUDA_CHECK."""
    r = subprocess.run([EULER_CLI + "_fp32"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Grid: 500 x 197 (with 2 ghost -> 504 x 201)" in r.stdout
    assert "Post-shock: rho=1.7755, p=159060.0, u=110.6272" in r.stdout


RIEMANN_CLI = os.path.join(ROOT, "precision-study_b200", "bin", "riemann2d_gpu")


def test_riemann_cli_rejects_an_unknown_configuration(pmhd_lib):
    r = subprocess.run([RIEMANN_CLI, "64", "5"], capture_output=True, text=True)
    assert r.returncode == 1 and "config_id must be 3, 6, or 12" in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_riemann_cli_without_device_exits_1(pmhd_lib):
    """The 2D Riemann drop-in prints the reference GPU program's header
    (riemann2d_gpu.cu:344-350) and, without a B200, exits with EXIT_FAILURE
    as the reference's CUDA_CHECK."""
    r = subprocess.run([RIEMANN_CLI + "_fp32", "64", "3"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Config:    cfg3_4shocks  (id=3)" in r.stdout and "Precision: fp32" in r.stdout
    assert "Grid:      64 x 64  dx=0.015625" in r.stdout and "T_end:     0.3" in r.stdout


RIEMANN1D_CLI = os.path.join(ROOT, "precision-study_b200", "bin", "riemann1d_gpu")


def test_riemann1d_cli_rejects_an_unknown_test(pmhd_lib):
    r = subprocess.run([RIEMANN1D_CLI, "200", "6"], capture_output=True, text=True)
    assert r.returncode == 1 and "test_id must be 1-5" in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_riemann1d_cli_without_device_exits_1(pmhd_lib):
    r = subprocess.run([RIEMANN1D_CLI + "_fp32", "200", "5", "hll"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Test:      Two_shocks  (id=5)" in r.stdout and "Solver:    HLL\n" in r.stdout
    assert "N=200  dx=0.005" in r.stdout
