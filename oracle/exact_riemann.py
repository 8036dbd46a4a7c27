"""Exact solution of the 1D Riemann problem for the ideal-gas Euler
equations (gamma = 1.4): Toro, "Riemann Solvers and Numerical Methods for
Fluid Dynamics", 3rd ed. (2009), chapter 4 -- star-region pressure by
Newton iteration on the pressure function (4.5)-(4.7) from the PV initial
guess, star velocity (4.9), and sampling of the wave pattern (section 4.5).

TEST INFRASTRUCTURE ONLY: the yardstick of the 1D Euler kernels' errors, as the
reference's analysis/euler/exact_riemann_errors.py is for its solvers.
"""
import math

import numpy as np

GAMMA = 1.4


def _f(p, rho, pk, a):
    """Pressure function f_K and its derivative for one side."""
    if p > pk:  # shock
        A = 2.0 / ((GAMMA + 1.0) * rho)
        B = (GAMMA - 1.0) / (GAMMA + 1.0) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + B))
    r = p / pk  # rarefaction
    return (2.0 * a / (GAMMA - 1.0)) * (r ** ((GAMMA - 1.0) / (2.0 * GAMMA)) - 1.0), \
        r ** (-(GAMMA + 1.0) / (2.0 * GAMMA)) / (rho * a)


def star_state(rl, ul, pl, rr, ur, pr, tol=1e-12):
    al, ar = math.sqrt(GAMMA * pl / rl), math.sqrt(GAMMA * pr / rr)
    p = max(1e-10, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (al + ar))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, al)
        fr, dr = _f(p, rr, pr, ar)
        p_new = max(1e-10, p - (fl + fr + ur - ul) / (dl + dr))
        change = abs(p_new - p) / (0.5 * (p_new + p))
        p = p_new
        if change < tol:
            break
    fl, _ = _f(p, rl, pl, al)
    fr, _ = _f(p, rr, pr, ar)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(ps, us, rl, ul, pl, rr, ur, pr, s):
    """(rho, u, p) at x/t = s."""
    g = GAMMA
    if s <= us:
        a = math.sqrt(g * pl / rl)
        if ps > pl:
            sl = ul - a * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
            if s <= sl:
                return rl, ul, pl
            return rl * (ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1), us, ps
        head = ul - a
        tail = us - a * (ps / pl) ** ((g - 1) / (2 * g))
        if s <= head:
            return rl, ul, pl
        if s >= tail:
            return rl * (ps / pl) ** (1 / g), us, ps
        c = 2 / (g + 1) + (g - 1) / ((g + 1) * a) * (ul - s)
        return rl * c ** (2 / (g - 1)), 2 / (g + 1) * (a + (g - 1) / 2 * ul + s), pl * c ** (2 * g / (g - 1))
    a = math.sqrt(g * pr / rr)
    if ps > pr:
        sr = ur + a * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
        if s >= sr:
            return rr, ur, pr
        return rr * (ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1), us, ps
    head = ur + a
    tail = us + a * (ps / pr) ** ((g - 1) / (2 * g))
    if s >= head:
        return rr, ur, pr
    if s <= tail:
        return rr * (ps / pr) ** (1 / g), us, ps
    c = 2 / (g + 1) - (g - 1) / ((g + 1) * a) * (ur - s)
    return rr * c ** (2 / (g - 1)), 2 / (g + 1) * (-a + (g - 1) / 2 * ur + s), pr * c ** (2 * g / (g - 1))


def solution(rl, ul, pl, rr, ur, pr, x0, t, x):
    ps, us = star_state(rl, ul, pl, rr, ur, pr)
    out = np.array([sample(ps, us, rl, ul, pl, rr, ur, pr, (xi - x0) / t) for xi in x])
    return out[:, 0], out[:, 1], out[:, 2]
