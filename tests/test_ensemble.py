"""Ensembles (pmhd_ensemble_*): many independent grids of uneven sizes
advanced by the same persistent stage launches.

The reference runs one grid per process (src/mhd/mhd2d_glm_gpu.cu main), so
the ensemble's oracle is the single-grid path itself: in the exact build every
member must end with exactly the bits a pmhd_solver run of that member gives
(which equal the reference CPU build -- test_gpu_parity.py); in the
performance build, within its parity tolerance.  The CPU
tests cover the seeded benchmark description, the periodic-band Brio-Wu
state it uses, and argument checking.
"""
import ctypes
import math

import numpy as np
import pytest

from test_abi import has_gpu

SLOPES = [(k, m) for k in range(5) for m in range(5) if k + m and math.gcd(k, m) == 1]


# ---- CPU: the seeded benchmark description --------------------------------

def test_default_description_is_seeded_and_prefix_stable(pmhd_lib):
    a = pmhd_lib.describe_ensemble(64, seed=7)
    b = pmhd_lib.describe_ensemble(64, seed=7)
    c = pmhd_lib.describe_ensemble(16, seed=7)
    d = pmhd_lib.describe_ensemble(64, seed=8)
    assert [m.as_dict() for m in a] == [m.as_dict() for m in b]
    assert [m.as_dict() for m in a[:16]] == [m.as_dict() for m in c]
    assert [m.as_dict() for m in a] != [m.as_dict() for m in d]


def test_default_description_follows_the_benchmark_recipe(pmhd_lib):
    ms = pmhd_lib.describe_ensemble(512, seed=0)
    sizes = [m.nx for m in ms]
    assert all(m.nx == m.ny for m in ms)
    assert set(sizes) == {64, 128, 256, 512}
    for s in (64, 128, 256, 512):  # uniform over four sizes: 128 expected each
        assert 80 < sizes.count(s) < 176
    slopes = set()
    for k, m in enumerate(ms):
        assert (m.x_min, m.x_max, m.y_min, m.y_max) == (0.0, 1.0, 0.0, 1.0)
        assert tuple(m.bc) == (0, 0, 0, 0)
        if k % 2 == 0:
            assert m.problem == pmhd_lib.PROBLEM_ORSZAG_TANG and m.gamma == 5.0 / 3.0
            assert m.t_end == 0.5 and m.nparams == 1
            assert 0.5 <= m.params[0] < 1.5
        else:
            assert m.problem == pmhd_lib.PROBLEM_BRIO_WU_TORUS and m.gamma == 2.0
            assert m.t_end == 0.1 and m.nparams == 2
            slopes.add((int(m.params[0]), int(m.params[1])))
    assert slopes <= set(SLOPES) and len(slopes) >= 10
    amps = np.array([m.params[0] for m in ms[0::2]])
    assert 0.9 < amps.mean() < 1.1


def test_default_description_snaps_the_angle_to_the_nearest_slope(pmhd_lib):
    """Odd member k draws u = the second of its three splitmix64 draws and
    uses the slope whose angle atan2(k, m) is nearest to u * pi / 2."""
    def splitmix64(x):
        x = (x + 0x9E3779B97F4A7C15) & (2 ** 64 - 1)
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2 ** 64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2 ** 64 - 1)
        return x, z ^ (z >> 31)

    ms = pmhd_lib.describe_ensemble(40, seed=11)
    st = 11
    for k in range(40):
        draws = []
        for _ in range(3):
            st, z = splitmix64(st)
            draws.append((z >> 11) / 2.0 ** 53)
        assert ms[k].nx == (64, 128, 256, 512)[min(3, int(draws[0] * 4))]
        if k % 2:
            ang = draws[1] * math.pi / 2
            want = min(SLOPES, key=lambda s: abs(math.atan2(s[0], s[1]) - ang))
            assert (ms[k].params[0], ms[k].params[1]) == want
        else:
            assert ms[k].params[0] == 0.5 + draws[1]


def test_default_description_rejects_bad_arguments(pmhd_lib):
    L = pmhd_lib.load()
    assert L.pmhd_ensemble_describe_default(-1, 0, None) == pmhd_lib.ERR_ARG
    assert L.pmhd_ensemble_describe_default(3, 0, None) == pmhd_lib.ERR_ARG
    assert L.pmhd_ensemble_describe_default(0, 0, None) == pmhd_lib.OK


# ---- CPU: the periodic-band Brio-Wu state ----------------------------------

@pytest.mark.parametrize("k,m", SLOPES)
def test_band_brio_wu_state_is_periodic_and_divergence_consistent(pmhd_lib, k, m):
    n = 64
    U = pmhd_lib.problem_state(pmhd_lib.PROBLEM_BRIO_WU_TORUS, [k, m], nx=n, ny=n, gamma=2.0)
    # The pattern repeats over the box: ghost cells equal the wrapped interior.
    np.testing.assert_array_equal(U[2:-2, 0:2], U[2:-2, n:n + 2])
    np.testing.assert_array_equal(U[2:-2, -2:], U[2:-2, 2:4])
    np.testing.assert_array_equal(U[0:2, 2:-2], U[n:n + 2, 2:-2])
    # Normal field 0.75 everywhere, tangential +-1, Brio-Wu densities.
    nrm = np.array([m, k], dtype=float) / math.hypot(k, m)
    bn = U[..., 5] * nrm[0] + U[..., 6] * nrm[1]
    bt = -U[..., 5] * nrm[1] + U[..., 6] * nrm[0]
    np.testing.assert_allclose(bn, 0.75, atol=1e-14)
    np.testing.assert_allclose(np.abs(bt), 1.0, atol=1e-14)
    left = U[..., 0] == 1.0
    assert np.all(left | (U[..., 0] == 0.125))
    assert np.all((bt > 0) == left)
    assert 0.4 < left[2:-2, 2:-2].mean() < 0.6


def test_band_brio_wu_rejects_bad_slopes(pmhd_lib):
    for params in ([0, 0], [1.5, 2], [-1, 1], [65, 1]):
        with pytest.raises(pmhd_lib.PmhdError):
            pmhd_lib.problem_state(pmhd_lib.PROBLEM_BRIO_WU_TORUS, params, nx=16, ny=16, gamma=2.0)


@pytest.mark.parametrize("k,m", SLOPES)
def test_band_brio_wu_runs_to_its_end_time_on_the_oracle(pmhd_lib, oracle, k, m):
    """Every slope the description can pick runs to t_end = 0.1 with the
    reference algorithm (oracle, fp64) at 64^2."""
    n = 64
    U = pmhd_lib.problem_state(pmhd_lib.PROBLEM_BRIO_WU_TORUS, [k, m], nx=n, ny=n, gamma=2.0)
    st = oracle.run("f64", oracle.make_config(n, n, 0.1, gamma=2.0), U)
    assert st.status == 0 and st.t == 0.1


def test_rotated_tube_against_walls_fails_at_the_wall_on_the_oracle(pmhd_lib, oracle):
    """Why the benchmark uses the periodic bands: a single interface at 0.8
    rad meeting zero-gradient walls drives the reference algorithm to a
    non-physical state in the wall column within a few steps."""
    n = 128
    U = pmhd_lib.problem_state(pmhd_lib.PROBLEM_BRIO_WU_2D, [0.8], nx=n, ny=n, gamma=2.0, bc=(2, 2, 2, 2))
    st = oracle.run("f64", oracle.make_config(n, n, 0.1, gamma=2.0, bc=(2, 2, 2, 2)), U)
    assert st.status == 3 and st.steps < 20 and st.bad_i <= 1


# ---- CPU: argument checking --------------------------------------------------

def _create_rc(pmhd_lib, members, **cfg):
    arr = (pmhd_lib.MemberDesc * len(members))(*members) if members else None
    c = pmhd_lib.make_config(**cfg)
    h = ctypes.c_void_p(1)
    rc = pmhd_lib.load().pmhd_ensemble_create(ctypes.byref(c), arr, len(members), ctypes.byref(h))
    if rc == pmhd_lib.OK:
        pmhd_lib.load().pmhd_ensemble_destroy(h)
    else:
        assert h.value is None
    return rc


def test_create_rejects_bad_members(pmhd_lib):
    ok = pmhd_lib.member(32, 32)
    assert _create_rc(pmhd_lib, []) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [ok, pmhd_lib.member(2, 32)]) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [pmhd_lib.member(32, 32, bc=(0, 1, 0, 0))]) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [pmhd_lib.member(32, 32, gamma=1.0)]) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [pmhd_lib.member(32, 32, domain=(1.0, 0.0, 0.0, 1.0))]) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [ok], cfl=1.5) == pmhd_lib.ERR_ARG
    assert _create_rc(pmhd_lib, [ok], steps_per_graph=3) == pmhd_lib.ERR_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly(pmhd_lib):
    assert _create_rc(pmhd_lib, [pmhd_lib.member(32, 32)]) == pmhd_lib.ERR_NODEVICE


def test_null_ensemble_handles_are_rejected(pmhd_lib):
    L = pmhd_lib.load()
    st = pmhd_lib.Stats()
    assert L.pmhd_ensemble_advance(None, -1, ctypes.byref(st)) == pmhd_lib.ERR_ARG
    assert L.pmhd_ensemble_member_stats(None, 0, ctypes.byref(st)) == pmhd_lib.ERR_ARG
    assert L.pmhd_ensemble_get_state(None, 0, None, 0) == pmhd_lib.ERR_ARG
    assert L.pmhd_ensemble_destroy(None) == pmhd_lib.OK


# ---- GPU: every member equals its single-grid run ---------------------------

def _mixed_members(pmhd_lib):
    m = pmhd_lib.member
    return [
        m(48, 32, t_end=0.06),
        m(40, 40, problem=pmhd_lib.PROBLEM_BRIO_WU_TORUS, params=(1, 2), gamma=2.0, t_end=0.05),
        m(64, 24, problem=pmhd_lib.PROBLEM_ORSZAG_TANG, params=(1.3,), t_end=0.04),
        m(36, 52, problem=pmhd_lib.PROBLEM_KH_REFLECT, params=(0.08, 0.1), domain=(0.0, 1.0, -1.0, 1.0),
          bc=(0, 0, 1, 1), t_end=0.2),
        m(33, 17, problem=pmhd_lib.PROBLEM_BRIO_WU_2D, params=(0.2,), gamma=2.0, bc=(2, 2, 2, 2), t_end=0.03),
        m(16, 16, t_end=0.02),
    ]


def _single(pmhd_lib, d, max_steps=-1, check=True, **common):
    with pmhd_lib.Solver(nx=d.nx, ny=d.ny, gamma=d.gamma, domain=(d.x_min, d.x_max, d.y_min, d.y_max),
                         bc=tuple(d.bc), **common) as s:
        s.init_problem(d.problem, list(d.params[:d.nparams]) if d.nparams else None)
        st = s.advance(t_end=d.t_end, max_steps=max_steps, check=check)
        return s.get_state(), st


COMMONS = [
    dict(precision="fp64", exact=True),
    dict(precision="mixed", exact=True),
    dict(precision="fp32", exact=False),
    dict(precision="mixed", exact=False, order="first", solver="hll"),
]


def _same(got, want, common, msg, exact_ref=None):
    """Exact build: bit for bit.  Performance build: the batched and the
    one-grid kernel instantiations may contract multiply-adds differently, so
    within the fast-build parity tolerances (fp64 1e-12, fp32 / mixed 1e-5 on
    the MHD variables) -- or, per variable, within a tenth of how far the
    one-grid performance run itself lies from the exact-build run
    (`exact_ref`), where rounding alone moves a member further than that bar
    (the reflecting-wall Kelvin-Helmholtz member in binary32: 1.8e-3 in my
    between the two builds, so two valid roundings differ by ~5e-5)."""
    if common.get("exact"):
        np.testing.assert_array_equal(got, want, err_msg=msg)
        return
    import pmhd
    tol = np.full(9, 1e-12 if common.get("precision") == "fp64" else 1e-5)
    if exact_ref is not None:
        own = pmhd.relative_l2(exact_ref.astype(np.float64), want.astype(np.float64))
        tol = np.maximum(tol, 0.1 * own)
    rel = pmhd.relative_l2(want.astype(np.float64), got.astype(np.float64))
    live = [0, 1, 2, 4, 5, 6]
    assert np.all(rel[live] < tol[live]), (msg, rel, tol)


@pytest.mark.gpu
@pytest.mark.parametrize("common", COMMONS, ids=lambda c: "-".join(str(v) for v in c.values()))
def test_members_equal_single_grid_runs(pmhd_lib, common):
    members = _mixed_members(pmhd_lib)
    with pmhd_lib.Ensemble(members, **common) as e:
        tot = e.advance()
        assert tot.status == pmhd_lib.OK
        zc = 0
        for k, d in enumerate(members):
            U, st = _single(pmhd_lib, d, **common)
            ms = e.member_stats(k)
            assert ms.zone_cycles == ms.steps * d.nx * d.ny
            zc += ms.zone_cycles
            if common.get("exact"):
                assert ms.steps == st.steps > 0 and ms.t == st.t, k
                assert (ms.x_evals, ms.y_evals, ms.degenerate, ms.nonphysical) == \
                    (st.x_evals, st.y_evals, st.degenerate, st.nonphysical), k
            else:
                assert abs(ms.steps - st.steps) <= 1 and ms.t == pytest.approx(st.t, rel=1e-12), k
            ref = None
            if not common.get("exact"):
                ref, _ = _single(pmhd_lib, d, **dict(common, exact=True))
            _same(e.get_state(k), U, common, f"member {k}", exact_ref=ref)
        assert tot.zone_cycles == zc
        assert tot.steps == max(e.member_stats(k).steps for k in range(len(members)))


@pytest.mark.gpu
def test_step_limited_advance_resumes_exactly(pmhd_lib):
    members = _mixed_members(pmhd_lib)
    common = dict(precision="fp64", exact=True, steps_per_graph=4)
    with pmhd_lib.Ensemble(members, **common) as e:
        tot = e.advance(max_steps=5)
        assert tot.status == pmhd_lib.OK
        for k, d in enumerate(members):
            assert e.member_stats(k).steps == 5
            U5, _ = _single(pmhd_lib, d, max_steps=5, **common)
            np.testing.assert_array_equal(e.get_state(k), U5)
        e.advance()
        for k, d in enumerate(members):
            U, st = _single(pmhd_lib, d, **common)
            assert e.member_stats(k).steps == st.steps
            np.testing.assert_array_equal(e.get_state(k), U)


@pytest.mark.gpu
def test_a_failing_member_halts_alone(pmhd_lib):
    """A member that reaches a non-physical state stops with its own status
    (as its single-grid run does); the others run to their end times."""
    members = _mixed_members(pmhd_lib)
    bad = pmhd_lib.member(128, 128, problem=pmhd_lib.PROBLEM_BRIO_WU_2D, params=(0.8,), gamma=2.0,
                          bc=(2, 2, 2, 2), t_end=0.1)
    members.insert(2, bad)
    common = dict(precision="fp64", exact=True)
    with pmhd_lib.Ensemble(members, **common) as e:
        tot = e.advance(check=False)
        assert tot.status == pmhd_lib.ERR_STAGE1
        Ub, sb = _single(pmhd_lib, bad, check=False, **common)
        mb = e.member_stats(2)
        assert mb.status == sb.status == pmhd_lib.ERR_STAGE1
        assert (mb.bad_i, mb.bad_j, mb.bad_step, mb.steps) == (sb.bad_i, sb.bad_j, sb.bad_step, sb.steps)
        assert (tot.bad_i, tot.bad_j) == (sb.bad_i, sb.bad_j)
        for k, d in enumerate(members):
            if k == 2:
                continue
            U, st = _single(pmhd_lib, d, **common)
            assert e.member_stats(k).status == pmhd_lib.OK and e.member_stats(k).steps == st.steps
            np.testing.assert_array_equal(e.get_state(k), U, err_msg=f"member {k}")
        # A later call leaves the failed member frozen and reports no new failure.
        tot2 = e.advance(max_steps=4)
        assert tot2.status == pmhd_lib.OK and e.member_stats(2).steps == sb.steps


@pytest.mark.gpu
def test_default_ensemble_with_autotuner_matches_single_runs(pmhd_lib):
    """Benchmark recipe (sizes capped to keep the single-grid runs short):
    whichever kernel variant the autotuner picks, every member agrees with
    its single-grid run (performance build: within its parity tolerance)."""
    ms = pmhd_lib.describe_ensemble(12, seed=3)
    for m in ms:
        m.nx = m.ny = min(m.nx, 128)
        m.t_end = 0.05 if m.problem == pmhd_lib.PROBLEM_ORSZAG_TANG else 0.02
    common = dict(precision="mixed", exact=False)
    with pmhd_lib.Ensemble(ms, autotune=True, **common) as e:
        tot = e.advance()
        assert tot.status == pmhd_lib.OK and tot.tile_height in (19, 8)
        for k, d in enumerate(ms):
            U, st = _single(pmhd_lib, d, **common)
            assert abs(e.member_stats(k).steps - st.steps) <= 1
            _same(e.get_state(k), U, common, f"member {k}")


@pytest.mark.gpu
def test_per_size_tuned_plan_is_bit_identical(pmhd_lib):
    """With autotune, each grid size is timed on its own and the sizes that
    choose the same tile height share a work list (one launch per chosen
    height and stage).  Whatever plan results, the exact build still gives
    every member the bits of its single-grid run, including members that
    took tuning steps while the others did not, and each member reports the
    tile height of its part."""
    m = pmhd_lib.member
    members = [m(64, 64, t_end=0.05), m(160, 160, t_end=0.03), m(64, 64, params=(1.2,), t_end=0.05),
               m(96, 40, problem=pmhd_lib.PROBLEM_BRIO_WU_TORUS, params=(1, 1), gamma=2.0, t_end=0.02),
               m(160, 160, params=(0.8,), t_end=0.03)]
    common = dict(precision="mixed", exact=True)
    with pmhd_lib.Ensemble(members, autotune=True, **common) as e:
        tot = e.advance()
        assert tot.status == pmhd_lib.OK
        heights = [e.member_stats(k).tile_height for k in range(len(members))]
        assert set(heights) <= {19, 8}
        assert heights[0] == heights[2] and heights[1] == heights[4]  # per size class
        for k, d in enumerate(members):
            U, st = _single(pmhd_lib, d, **common)
            ms = e.member_stats(k)
            assert ms.steps == st.steps and ms.t == st.t, k
            assert (ms.degenerate, ms.nonphysical) == (st.degenerate, st.nonphysical), k
            np.testing.assert_array_equal(e.get_state(k), U, err_msg=f"member {k}")
