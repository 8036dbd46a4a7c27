"""ctypes bindings for the CPU oracle (oracle/liboracle.so).

Test infrastructure only: the oracle is the checker, never the thing under
test or the product path.  It restates the reference's serial solver
(src/mhd/mhd2d_glm_cpu.cpp + include/mhd/*.hpp) in C, plus this project's
mixed-precision variant.
"""
import ctypes
import hashlib
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

BC_PERIODIC, BC_REFLECT, BC_TRANSMISSIVE = 0, 1, 2
PROBLEM_OT, PROBLEM_KH_REF = 0, 1


class OrConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("hlld_tol", ctypes.c_double),
        ("cfl", ctypes.c_double), ("alpha", ctypes.c_double),
        ("t_end", ctypes.c_double),
        ("use_muscl", ctypes.c_int), ("use_hlld", ctypes.c_int),
        ("bc", ctypes.c_int * 4),
        ("max_steps", ctypes.c_int),
    ]


class OrStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int), ("status", ctypes.c_int),
        ("bad_i", ctypes.c_int), ("bad_j", ctypes.c_int),
        ("t", ctypes.c_double), ("ch_last", ctypes.c_double),
        ("x_evals", ctypes.c_ulonglong), ("y_evals", ctypes.c_ulonglong),
        ("degenerate", ctypes.c_ulonglong), ("nonphysical", ctypes.c_ulonglong),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        dp, fp = P(ctypes.c_double), P(ctypes.c_float)
        for name, ptr in (("f64", dp), ("f32", fp), ("mixed", dp)):
            fn = getattr(_lib, "or_run_" + name)
            fn.argtypes = [P(OrConfig), ptr, P(OrStats)]
            fn.restype = ctypes.c_int
        fn = _lib.or_run_hancock_mixed
        fn.argtypes = [P(OrConfig), dp, P(OrStats)]
        fn.restype = ctypes.c_int
        for name, ptr in (("f64", dp), ("f32", fp)):
            fn = getattr(_lib, "or_run_hancock_" + name)
            fn.argtypes = [P(OrConfig), ptr, P(OrStats)]
            fn.restype = ctypes.c_int
            fn = getattr(_lib, "or_init_ref_problem_" + name)
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 5 + [ptr]
            fn.restype = None
            fn = getattr(_lib, "or_write_dat_lines_" + name)
            fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 5 + [ptr]
            fn.restype = ctypes.c_int
            fn = getattr(_lib, "or_fill_ghosts_" + name)
            fn.argtypes = [P(OrConfig), ptr]
            fn.restype = None
            fn = getattr(_lib, "or_point_hlld_" + name)
            fn.argtypes = [ptr, ptr, ptr, ctypes.c_int, ctypes.c_double, ctypes.c_double]
            fn.restype = ctypes.c_int
            fn = getattr(_lib, "or_point_glm_flux_" + name)
            fn.argtypes = [ptr, ptr, ctypes.c_double, ctypes.c_int, ctypes.c_int, ptr,
                           ctypes.c_double, ctypes.c_double]
            fn.restype = ctypes.c_int
            fn = getattr(_lib, "or_point_hll_" + name)
            fn.argtypes = [ptr, ptr, ptr, ctypes.c_int, ctypes.c_double]
            fn.restype = None
            fn = getattr(_lib, "or_point_cons_to_prim_" + name)
            fn.argtypes = [ptr, ptr, ctypes.c_double]
            fn.restype = None
            fn = getattr(_lib, "or_point_prim_to_cons_" + name)
            fn.argtypes = [ptr, ptr, ctypes.c_double]
            fn.restype = None
            fn = getattr(_lib, "or_point_fast_speed_" + name)
            fn.argtypes = [ptr, ctypes.c_int, ctypes.c_double]
            fn.restype = ctypes.c_double if name == "f64" else ctypes.c_float
            fn = getattr(_lib, "or_point_recon_" + name)
            fn.argtypes = [ptr] * 5
            fn.restype = None
            ct = ctypes.c_double if name == "f64" else ctypes.c_float
            fn = getattr(_lib, "or_point_minmod_" + name)
            fn.argtypes = [ct, ct]
            fn.restype = ct
            fn = getattr(_lib, "or_point_positive_" + name)
            fn.argtypes = [ptr, ctypes.c_double]
            fn.restype = ctypes.c_int
    return _lib


def dtype_of(prec):
    return np.float32 if prec == "f32" else np.float64


def _ptr(a):
    ct = ctypes.c_float if a.dtype == np.float32 else ctypes.c_double
    return a.ctypes.data_as(ctypes.POINTER(ct))


def make_config(nx, ny, t_end, cfl=0.25, alpha=0.18, muscl=True, hlld=True,
                gamma=5.0 / 3.0, tol=1e-4, domain=(0.0, 1.0, 0.0, 1.0),
                bc=(0, 0, 0, 0), max_steps=-1):
    c = OrConfig()
    c.nx, c.ny = nx, ny
    c.x_min, c.x_max, c.y_min, c.y_max = domain
    c.gamma, c.hlld_tol, c.cfl, c.alpha, c.t_end = gamma, tol, cfl, alpha, t_end
    c.use_muscl, c.use_hlld = int(muscl), int(hlld)
    for k in range(4):
        c.bc[k] = bc[k]
    c.max_steps = max_steps
    return c


def init_ref_problem(prec, problem, nx, ny, domain=(0.0, 1.0, 0.0, 1.0), gamma=5.0 / 3.0):
    """Ghosted AoS state of the reference's OT (problem 0) or KH (problem 1) IC."""
    dt = np.float32 if prec == "f32" else np.float64
    U = np.zeros((ny + 4, nx + 4, 9), dtype=dt)
    fn = getattr(lib(), "or_init_ref_problem_" + ("f32" if prec == "f32" else "f64"))
    fn(problem, nx, ny, *domain, gamma, _ptr(U))
    return U


def run(prec, cfg, U, t0=0.0, steps0=0, hancock=False):
    """Advance the ghosted AoS state U in place.  prec: f64 | f32 | mixed,
    SSPRK2 or (hancock=True) the MUSCL-Hancock variant."""
    st = OrStats()
    st.t, st.steps = t0, steps0
    fn = getattr(lib(), ("or_run_hancock_" if hancock else "or_run_") + prec)
    assert U.dtype == (np.float32 if prec == "f32" else np.float64)
    assert U.flags["C_CONTIGUOUS"] and U.shape == (cfg.ny + 4, cfg.nx + 4, 9)
    fn(ctypes.byref(cfg), _ptr(U), ctypes.byref(st))
    return st


def fill_ghosts(prec, cfg, U):
    getattr(lib(), "or_fill_ghosts_" + ("f32" if prec == "f32" else "f64"))(ctypes.byref(cfg), _ptr(U))


def dat_lines_md5(prec, cfg, U, path):
    fn = getattr(lib(), "or_write_dat_lines_" + ("f32" if prec == "f32" else "f64"))
    rc = fn(path.encode(), cfg.nx, cfg.ny, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max,
            cfg.gamma, _ptr(U))
    assert rc == 0
    with open(path, "rb") as f:
        return hashlib.md5(f.read()).hexdigest()


def data_lines_md5_of_file(path):
    """md5 of the non-'#' lines of a .dat file (the reference's regression gate)."""
    h = hashlib.md5()
    with open(path, "rb") as f:
        for line in f:
            if not line.startswith(b"#"):
                h.update(line)
    return h.hexdigest()
