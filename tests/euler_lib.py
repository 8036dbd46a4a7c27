"""ctypes access to the Euler oracle (oracle/euler_oracle.h via
oracle/liboracle.so) and formatting of its results in the reference's .dat
format.  Test infrastructure only."""
import ctypes
import hashlib
import os

import numpy as np

import oracle_lib


def _lib():
    return oracle_lib.lib()


def _ctype(prec):
    return ctypes.c_double if prec == "fp64" else ctypes.c_float


def _np(prec):
    return np.float64 if prec == "fp64" else np.float32


def riemann2d(n, config, solver="hllc", prec="fp64", t_end=-1.0, max_steps=-1, ny=None):
    """Oracle 2D Riemann run on n x ny (default n x n): (steps, t, prims [ny][n][4])."""
    T = _ctype(prec)
    ny = n if ny is None else ny
    fn = getattr(_lib(), "eo_riemann2d_" + ("f64" if prec == "fp64" else "f32"))
    fn.restype = ctypes.c_longlong
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, T, ctypes.c_longlong, ctypes.c_void_p,
                   ctypes.POINTER(T)]
    out = np.zeros((ny, n, 4), dtype=_np(prec))
    t = T()
    steps = fn(n, ny, config, 1 if solver == "hll" else 0, T(t_end), max_steps, out.ctypes.data, ctypes.byref(t))
    assert steps >= 0
    return steps, t.value, out


def shock_bubble(nx=500, ny=197, solver="hllc", prec="fp64", t_end=-1.0, max_steps=-1):
    """Oracle shock-bubble run (src/euler/euler2d_cpu.cpp) on nx x ny:
    (steps, t, prims [ny][nx][4])."""
    T = _ctype(prec)
    fn = getattr(_lib(), "eo_shock_bubble_" + ("f64" if prec == "fp64" else "f32"))
    fn.restype = ctypes.c_longlong
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p,
                   ctypes.POINTER(T)]
    out = np.zeros((ny, nx, 4), dtype=_np(prec))
    t = T()
    steps = fn(nx, ny, 1 if solver == "hll" else 0, t_end, max_steps, out.ctypes.data, ctypes.byref(t))
    assert steps >= 0
    return steps, t.value, out


def riemann1d(n, test, solver="hllc", prec="fp64"):
    """Oracle 1D Riemann run: (steps, t, [n][3] = rho, u, p)."""
    T = _ctype(prec)
    fn = getattr(_lib(), "eo_riemann1d_" + ("f64" if prec == "fp64" else "f32"))
    fn.restype = ctypes.c_longlong
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(T)]
    out = np.zeros((n, 3), dtype=_np(prec))
    t = T()
    steps = fn(n, test, 1 if solver == "hll" else 0, out.ctypes.data, ctypes.byref(t))
    assert steps >= 0
    return steps, t.value, out


def _fmt(prec):
    return "%.17e" if prec == "fp64" else "%.9e"


def dat_md5_2d(prims, prec):
    """md5 of the .dat file src/euler/riemann2d_cpu.cpp:313-325 writes."""
    n = prims.shape[0]
    T = _np(prec)
    dx = T(T(1.0) - T(0.0)) / T(n)
    f = _fmt(prec)
    lines = []
    for j in range(n):
        y = T(0.0) + (T(j) + T(0.5)) * dx
        for i in range(n):
            x = T(0.0) + (T(i) + T(0.5)) * dx
            vals = (x, y) + tuple(prims[j, i])
            lines.append(" ".join(f % float(v) for v in vals) + "\n")
    return hashlib.md5("".join(lines).encode()).hexdigest()


def dat_md5_shock_bubble(prims, prec):
    """md5 of the data lines (those not starting with '#') of the .dat file
    src/euler/euler2d_cpu.cpp:378-394 writes: x outermost, one line per cell
    (x y rho u v p), a blank line after each column; cell centres are
    binary64 expressions (config.hpp literals) stored in the precision's
    type."""
    ny, nx = prims.shape[:2]
    T = _np(prec)
    dx = float(T(T(0.225 - 0.0) / T(nx)))
    dy = float(T(T(0.089 - 0.0) / T(ny)))
    f = _fmt(prec)
    ys = [f % float(T(0.0 + (j + 0.5) * dy)) for j in range(ny)]
    lines = []
    for i in range(nx):
        x = f % float(T(0.0 + (i + 0.5) * dx))
        for j in range(ny):
            lines.append(x + " " + ys[j] + " " + " ".join(f % float(v) for v in prims[j, i]) + "\n")
        lines.append("\n")
    return hashlib.md5("".join(lines).encode()).hexdigest()


def dat_md5_1d(out, prec):
    """md5 of the .dat file src/euler/riemann1d_cpu.cpp:203-210 writes."""
    n = out.shape[0]
    T = _np(prec)
    dx = T(T(1.0) - T(0.0)) / T(n)
    f = _fmt(prec)
    lines = []
    for i in range(n):
        x = T(0.0) + T(i + 0.5) * dx
        lines.append(" ".join(f % float(v) for v in (x,) + tuple(out[i])) + "\n")
    return hashlib.md5("".join(lines).encode()).hexdigest()
