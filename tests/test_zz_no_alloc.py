"""GPU test of pmhd_advance_noalloc, the time loop for callers that must not
allocate device memory while they run (a process that pre-carves all GPU
memory into its own pool, an allocator hook that forbids cudaMalloc after
start-up).  It works on the caller's device buffers and keeps its working
state in one fixed array compiled into the library, shared by every call.

Checked against the regular handle path (pmhd_create / pmhd_set_state /
pmhd_advance / pmhd_get_state) on the same inputs: both run the same
kernels, so the results must agree bit for bit (exact and fast builds).
Several calls in a row, with different problems and precisions, show that
what one call leaves in the shared array does not leak into the next.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(pmhd, U, t_end, max_steps=-1, t0=0.0, step0=0, in_place=False, **cfg_kwargs):
    import torch

    cfg = pmhd.make_config(**cfg_kwargs)
    d_in = torch.from_numpy(np.ascontiguousarray(U)).cuda()  # the caller's own device buffers
    d_out = d_in if in_place else torch.empty_like(d_in)
    st = pmhd.Stats()
    rc = pmhd.load().pmhd_advance_noalloc(ctypes.byref(cfg), d_in.data_ptr(), d_out.data_ptr(), t0, step0, t_end,
                                          max_steps, None, ctypes.byref(st))
    torch.cuda.synchronize()
    return rc, d_out.cpu().numpy(), st


def _regular(pmhd, U, t_end, max_steps=-1, **cfg_kwargs):
    with pmhd.Solver(**cfg_kwargs) as s:
        s.set_state(U)
        st = s.advance(t_end=t_end, max_steps=max_steps)
        return s.get_state(), st


def _interior(pmhd, problem, params=None, **cfg_kwargs):
    return np.ascontiguousarray(pmhd.problem_state(problem, params, **cfg_kwargs)[2:-2, 2:-2, :])


CASES = [
    # (problem, params, config, t_end, max_steps)
    (0, None, dict(nx=64, ny=48, precision="fp64", exact=True), 0.05, -1),
    (1, None, dict(nx=40, ny=40, precision="mixed", exact=True), 0.03, -1),
    (2, [0.08, 0.1], dict(nx=48, ny=36, precision="fp32", exact=False, domain=(0.0, 1.0, -1.0, 1.0),
                          bc=(0, 0, 1, 1)), 1.0, 11),
    (0, None, dict(nx=64, ny=48, precision="mixed", exact=False), 0.04, -1),
]


def test_noalloc_matches_regular_path_over_consecutive_calls(pmhd_lib):
    first = None
    for problem, params, cfg, t_end, max_steps in CASES:
        U0 = _interior(pmhd_lib, problem, params, **cfg)
        rc, Un, sn = _noalloc(pmhd_lib, U0, t_end, max_steps, **cfg)
        assert rc == pmhd_lib.OK, pmhd_lib.strerror(rc)
        Ur, sr = _regular(pmhd_lib, U0, t_end, max_steps, **cfg)
        assert sn.steps == sr.steps > 0
        assert sn.t == sr.t and sn.ch_last == sr.ch_last
        assert (sn.degenerate, sn.nonphysical) == (sr.degenerate, sr.nonphysical)
        assert (sn.x_evals, sn.y_evals) == (sr.x_evals, sr.y_evals)
        np.testing.assert_array_equal(Un, Ur)
        if first is None:
            first = (U0, Un)
    # The first case again, after the array held other grids: same bits.
    U0, Un = first
    rc, again, _ = _noalloc(pmhd_lib, U0, CASES[0][3], **CASES[0][2])
    assert rc == pmhd_lib.OK
    np.testing.assert_array_equal(again, Un)


def test_noalloc_resume_in_place(pmhd_lib):
    """Two calls continuing one run in the caller's buffer (in place) equal
    one regular run."""
    cfg = dict(nx=56, ny=56, precision="fp64", exact=True)
    U0 = _interior(pmhd_lib, 0, **cfg)
    rc, U1, s1 = _noalloc(pmhd_lib, U0, 0.05, 9, in_place=True, **cfg)
    assert rc == pmhd_lib.OK and s1.steps == 9
    rc, U2, s2 = _noalloc(pmhd_lib, U1, 0.05, t0=s1.t, step0=s1.steps, in_place=True, **cfg)
    assert rc == pmhd_lib.OK
    Ur, sr = _regular(pmhd_lib, U0, 0.05, **cfg)
    assert s2.steps == sr.steps and s2.t == sr.t
    np.testing.assert_array_equal(U2, Ur)


def test_noalloc_second_call_leaves_device_memory_unchanged(pmhd_lib):
    """The entry point's promise: once the first call on a device has loaded
    the library's device code (which places the fixed array in device
    memory), a call allocates nothing.  Free device memory (cudaMemGetInfo,
    through torch.cuda.mem_get_info) is read before and after a second call
    with the same configuration, with the caller's buffers allocated up
    front."""
    import torch

    cfg_kwargs = dict(nx=96, ny=80, precision="mixed", exact=False)
    U0 = _interior(pmhd_lib, 0, **cfg_kwargs)
    cfg = pmhd_lib.make_config(**cfg_kwargs)
    d_in = torch.from_numpy(U0).cuda()
    d_out = torch.empty_like(d_in)
    lib = pmhd_lib.load()
    st = pmhd_lib.Stats()

    def call():
        rc = lib.pmhd_advance_noalloc(ctypes.byref(cfg), d_in.data_ptr(), d_out.data_ptr(), 0.0, 0, 0.05, -1,
                                      None, ctypes.byref(st))
        torch.cuda.synchronize()
        return rc

    assert call() == pmhd_lib.OK  # first call on this device: sets up, may load code
    first = d_out.cpu().numpy()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert call() == pmhd_lib.OK
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)
    np.testing.assert_array_equal(d_out.cpu().numpy(), first)
    assert st.steps > 0


def test_noalloc_rejects_grids_beyond_the_fixed_scratch(pmhd_lib):
    cfg = pmhd_lib.make_config(nx=1024, ny=1024, precision="fp64")
    st = pmhd_lib.Stats()
    big = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = pmhd_lib.load().pmhd_advance_noalloc(ctypes.byref(cfg), big, big, 0.0, 0, 0.1, 1, None, ctypes.byref(st))
    assert rc == pmhd_lib.ERR_UNSUPPORTED
    no = pmhd_lib.make_config(nx=587, ny=587, precision="fp64")
    assert pmhd_lib.load().pmhd_advance_noalloc(ctypes.byref(no), big, big, 0.0, 0, 0.1, 1, None,
                                                ctypes.byref(st)) == pmhd_lib.ERR_UNSUPPORTED
    U0 = _interior(pmhd_lib, 0, nx=586, ny=586, precision="fp64")
    rc, _, s = _noalloc(pmhd_lib, U0, 1.0, 2, nx=586, ny=586, precision="fp64")
    assert rc == pmhd_lib.OK and s.steps == 2
