"""Exact solution of the Sod shock tube (ideal gas, gamma = 1.4):
the classical two-rarefaction/shock Riemann solution with Newton iteration on the
star pressure (E. F. Toro, "Riemann Solvers and Numerical Methods for Fluid
Dynamics", ch. 4), for error measurements of shock-tube runs."""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho_k, p_k, c_k, g):
    if p > p_k:  # shock
        A = 2.0 / ((g + 1.0) * rho_k)
        B = (g - 1.0) / (g + 1.0) * p_k
        q = math.sqrt(A / (p + B))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (p + B))
    r = p / p_k  # rarefaction
    return 2.0 * c_k / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0), 1.0 / (rho_k * c_k) * r ** (-(g + 1.0) / (2.0 * g))


def sod_exact(x: np.ndarray, t: float, g: float = 1.4, x0: float = 0.5,
              left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)) -> np.ndarray:
    """Density of the exact solution at positions x and time t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = 0.5 * (pl + pr)
    for _ in range(50):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(p - dp, 1e-12)
        if abs(dp) < 1e-14:
            break
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    out = np.empty_like(x, dtype=float)
    s = (x - x0) / t
    # left rarefaction (p* < pl for Sod)
    rls = rl * (p / pl) ** (1.0 / g)
    cls = cl * (p / pl) ** ((g - 1.0) / (2.0 * g))
    shl, stl = ul - cl, u - cls
    # right shock
    rrs = rr * ((p / pr + (g - 1.0) / (g + 1.0)) / ((g - 1.0) / (g + 1.0) * p / pr + 1.0))
    sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * p / pr + (g - 1.0) / (2.0 * g))
    fan = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * (ul - s))
    rho_fan = rl * (np.maximum(fan, 0.0) / cl) ** (2.0 / (g - 1.0))
    out[:] = np.where(s < shl, rl, np.where(s < stl, rho_fan, np.where(s < u, rls, np.where(s < sr, rrs, rr))))
    return out
