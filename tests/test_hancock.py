"""The 2D MUSCL-Hancock variant (order "hancock"): one predictor-corrector
stage per step.  No 2D reference exists, so the oracle (or_run_hancock,
oracle/oracle_step.h; the mixed policy's or_run_hancock_mixed,
oracle/pmhd_oracle.c) is the unsplit 2D form of the reference's 1D Hancock
predictor on the 2D solver's own pinned building blocks; parity is GPU vs
that oracle (bit for bit in the exact build).  CPU tests check the oracle's
conservation, its agreement with the SSPRK2 scheme at second order, and the
mixed policy against binary64.
"""
import numpy as np
import pytest

from test_gpu_parity import PREC_OF, gpu_run, interior, oracle_run  # noqa: F401


def _oracle_hancock(oracle, prec, nx, ny, t_end, solver="hlld", problem=0, max_steps=-1, bc=(0, 0, 0, 0),
                    domain=(0.0, 1.0, 0.0, 1.0), gamma=5.0 / 3.0, U0=None):
    cfg = oracle.make_config(nx, ny, t_end, hlld=(solver == "hlld"), gamma=gamma, domain=domain, bc=bc,
                             max_steps=max_steps)
    if U0 is None:
        U = oracle.init_ref_problem("f32" if prec == "fp32" else "f64", problem, nx, ny, domain, gamma)
    else:
        U = np.array(U0, copy=True)
    st = oracle.run(PREC_OF[prec], cfg, U, hancock=True)
    return U, st


# ---- CPU ---------------------------------------------------------------------

def test_oracle_hancock_conserves_and_tracks_ssprk2(oracle):
    nx = ny = 64
    U0 = oracle.init_ref_problem("f64", 0, nx, ny)
    Uh, sh = _oracle_hancock(oracle, "fp64", nx, ny, 0.2)
    Us, ss = oracle_run(oracle, "fp64", nx, ny, 0.2)
    assert sh.status == 0 and sh.t == pytest.approx(0.2)
    for k in (0, 1, 2, 4, 5, 6):  # periodic box: totals of conserved fields
        assert abs(interior(Uh)[..., k].sum() - interior(U0)[..., k].sum()) < 1e-10 * max(1.0, np.abs(U0[..., k]).sum())
    rel = np.sqrt(np.mean((interior(Uh) - interior(Us)) ** 2, axis=(0, 1))) / \
        np.sqrt(np.mean(interior(Us) ** 2, axis=(0, 1)) + 1e-300)
    assert np.all(rel[[0, 1, 2, 4, 5, 6]] < 1e-2), rel


def test_oracle_hancock_converges_at_second_order(oracle):
    """Smooth problem (Orszag-Tang before shocks form, t = 0.05): the error
    against a 4x finer Hancock run, restricted, falls by ~4x per refinement."""
    def run(n):
        U, _ = _oracle_hancock(oracle, "fp64", n, n, 0.05)
        return interior(U)

    ref = run(256)
    errs = []
    for n in (32, 64):
        f = 256 // n
        r = ref.reshape(n, f, n, f, 9).mean(axis=(1, 3))
        errs.append(np.sqrt(np.mean((run(n)[..., 0] - r[..., 0]) ** 2)))
    assert errs[0] / errs[1] > 3.0, errs


def test_oracle_hancock_mixed_tracks_fp64(oracle):
    """Mixed policy (binary32 faces, predictor and fluxes; binary64 recovery
    and update) against binary64 on a smooth Orszag-Tang run: conserved totals
    kept to binary64 round-off, per-variable relative L2 at binary32 level."""
    nx = ny = 64
    U0 = oracle.init_ref_problem("f64", 0, nx, ny)
    Um, sm = _oracle_hancock(oracle, "mixed", nx, ny, 0.1)
    Ud, sd = _oracle_hancock(oracle, "fp64", nx, ny, 0.1)
    assert sm.status == sd.status == 0 and sm.steps == sd.steps > 0
    for k in (0, 1, 2, 4, 5, 6):
        assert abs(interior(Um)[..., k].sum() - interior(U0)[..., k].sum()) < 1e-10 * max(1.0, np.abs(U0[..., k]).sum())
    rel = np.sqrt(np.mean((interior(Um) - interior(Ud)) ** 2, axis=(0, 1))) / \
        np.sqrt(np.mean(interior(Ud) ** 2, axis=(0, 1)) + 1e-300)
    assert np.all(rel[[0, 1, 2, 4, 5, 6]] < 1e-5), rel
    assert np.all(rel[[0, 1, 2, 4, 5, 6]] > 0.0), rel  # the binary32 stages are really used


# ---- GPU ---------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("solver", ["hlld", "hll"])
def test_hancock_exact_bitwise_vs_oracle_ot(pmhd_lib, oracle, prec, solver):
    nx, ny, t_end = 40, 24, 0.06
    Ug, sg = gpu_run(pmhd_lib, prec, nx, ny, t_end, order="hancock", solver=solver)
    Uo, so = _oracle_hancock(oracle, prec, nx, ny, t_end, solver=solver)
    assert sg.status == 0 and so.status == 0
    assert sg.steps == so.steps > 0 and sg.t == so.t and sg.ch_last == so.ch_last
    assert (sg.degenerate, sg.nonphysical) == (so.degenerate, so.nonphysical)
    assert (sg.x_evals, sg.y_evals) == (so.x_evals, so.y_evals)
    np.testing.assert_array_equal(Ug, Uo)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_hancock_exact_bitwise_walls_and_partial_tiles(pmhd_lib, oracle, prec):
    """KH with reflecting y walls on a 50 x 36 grid (partial tiles in x and
    y), and the rotated Brio-Wu tube with transmissive walls."""
    cases = [
        dict(nx=50, ny=36, t_end=0.2, problem=pmhd_lib.PROBLEM_KH_REFLECT, params=[0.08, 0.1],
             domain=(0.0, 1.0, -1.0, 1.0), bc=(0, 0, 1, 1), gamma=5.0 / 3.0),
        dict(nx=45, ny=33, t_end=0.04, problem=pmhd_lib.PROBLEM_BRIO_WU_2D, params=[0.3],
             domain=(0.0, 1.0, 0.0, 1.0), bc=(2, 2, 2, 2), gamma=2.0),
    ]
    for c in cases:
        U0 = pmhd_lib.problem_state(c["problem"], c["params"], nx=c["nx"], ny=c["ny"], precision=prec,
                                    domain=c["domain"], bc=c["bc"], gamma=c["gamma"])
        Ug, sg = gpu_run(pmhd_lib, prec, c["nx"], c["ny"], c["t_end"], order="hancock", domain=c["domain"],
                         bc=c["bc"], gamma=c["gamma"], U0=U0)
        Uo, so = _oracle_hancock(oracle, prec, c["nx"], c["ny"], c["t_end"], bc=c["bc"], domain=c["domain"],
                                 gamma=c["gamma"], U0=U0)
        assert sg.status == so.status == 0
        assert sg.steps == so.steps > 0 and sg.t == so.t
        assert (sg.degenerate, sg.nonphysical) == (so.degenerate, so.nonphysical)
        np.testing.assert_array_equal(Ug, Uo)


@pytest.mark.gpu
def test_hancock_step_limited_runs_resume_exactly(pmhd_lib, oracle):
    nx, ny = 48, 40
    Uo, so = _oracle_hancock(oracle, "fp64", nx, ny, 0.08)
    with pmhd_lib.Solver(nx=nx, ny=ny, precision="fp64", exact=True, order="hancock", steps_per_graph=4) as s:
        s.init_problem(0)
        assert s.advance(t_end=0.08, max_steps=7).steps == 7
        st = s.advance(t_end=0.08)
        U = s.get_state(layout=pmhd_lib.LAYOUT_GHOSTED)
    assert st.steps == so.steps and st.t == so.t
    np.testing.assert_array_equal(U, Uo)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5), ("mixed", 1e-5)])
def test_hancock_fast_build_close_to_the_oracle(pmhd_lib, oracle, prec, tol):
    nx = ny = 96
    Ug, sg = gpu_run(pmhd_lib, prec, nx, ny, 0.05, exact=False, order="hancock")
    Uo, so = _oracle_hancock(oracle, prec, nx, ny, 0.05)
    assert sg.steps == so.steps
    rel = pmhd_lib.relative_l2(interior(Uo).astype(np.float64), interior(Ug).astype(np.float64))
    assert np.all(rel[:8][[0, 1, 2, 4, 5, 6]] < tol), rel
