"""Shared helpers of the test suite: seeded physical states and error norms."""
from __future__ import annotations

import numpy as np

from fr_sdg_b200 import _abi as A

# Tolerance of the FP64 GPU path against the oracle: max|gpu - oracle| / max|oracle|.
TOL_FP64 = 1e-12
# Complex-step JVP.  Where a slip wall or a symmetric state makes the two wave
# speeds of smooth_max tie, the argument of smooth_abs is rounding noise x ~ 1e-16
# and its derivative x / sqrt(x^2 + 1e-14) ~ x / 1e-7 amplifies that noise by 1e7
# (macro_and_libc.hpp:80-102), so two correct implementations differ there at the
# 1e-11 level; elsewhere they agree to ~1e-15.
TOL_JVP = 1e-10
# FP32 residual (mixed-precision form) against the FP64 oracle on the same (rounded)
# state: each residual value sums O(N) products and a few quotients and square roots of
# O(1) quantities, so the FP32 result carries a few units of 2^-24 = 6e-8 relative to
# the largest terms; 5e-5 of max|R| leaves room for the cancellation inside the Riemann
# fluxes of discontinuous random states.
TOL_FP32 = 5e-5


def rel_err(got, ref) -> float:
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.max(np.abs(ref))
    if scale == 0.0:
        return float(np.max(np.abs(got)))
    return float(np.max(np.abs(got - ref)) / scale)


def gas_rhoE(cfg, rho, vel2, p):
    if cfg.gas_law == A.GAS_IDEAL:
        return p / (cfg.gamma - 1.0) + 0.5 * rho * vel2
    a, b = cfg.vdw_a, cfg.vdw_b
    ars = a * rho * rho
    return ((p + ars) * (1.0 - b * rho)) / (cfg.gamma - 1.0) - ars + 0.5 * rho * vel2


def random_state(cfg, seed: int, amp: float = 0.4, smooth: bool = False) -> np.ndarray:
    """Seeded physical state (positive density and pressure) in the DMDA layout.
    smooth=False draws every node independently (discontinuous traces, every
    Riemann branch); smooth=True perturbs a constant state per element."""
    rng = np.random.default_rng(seed)
    n = cfg.poly_deg + 1
    if cfg.dim == 2:
        nodes = cfg.n_elems[0] * cfg.n_elems[1] * n * n
    else:
        nodes = cfg.n_elems[0] * n
    if smooth:
        base = rng.uniform(-1, 1, size=4)
        jitter = rng.uniform(-1, 1, size=(nodes, 4)) * 0.05
        r = base[None, :] + jitter
    else:
        r = rng.uniform(-1, 1, size=(nodes, 4))
    rho = 1.0 + amp * r[:, 0]
    u = 0.8 * amp * r[:, 1]
    v = 0.8 * amp * r[:, 2] if cfg.dim == 2 else np.zeros(nodes)
    p = 1.0 + amp * r[:, 3]
    E = gas_rhoE(cfg, rho, u * u + v * v, p)
    if cfg.dim == 2:
        return np.stack([rho, rho * u, rho * v, E], axis=1).reshape(-1)
    N = cfg.n_elems[0]
    fields = np.stack([rho, rho * u, E], axis=0).reshape(3, N, n)  # eq, elem, node
    return np.ascontiguousarray(fields.transpose(1, 0, 2)).reshape(-1)


def cons_to_prim(cfg, U: np.ndarray) -> np.ndarray:
    """(log rho, u, [v], log e) of a conservative vector (problem_def.hpp:56-70)."""
    n = cfg.poly_deg + 1
    if cfg.dim == 2:
        q = U.reshape(-1, 4)
        rho = q[:, 0]
        u, v = q[:, 1] / rho, q[:, 2] / rho
        e = q[:, 3] / rho - 0.5 * (u * u + v * v)
        return np.stack([np.log(rho), u, v, np.log(e)], axis=1).reshape(-1)
    q = U.reshape(-1, 3, n)
    rho = q[:, 0]
    u = q[:, 1] / rho
    e = q[:, 2] / rho - 0.5 * u * u
    return np.stack([np.log(rho), u, np.log(e)], axis=1).reshape(-1)


def poisoned_state(cfg, seed: int, every: int = 3, gain: float = 4.0) -> np.ndarray:
    """A seeded state whose cell averages are admissible but whose nodes are not in
    every `every`-th element: there the deviations from the element's plain node mean
    are amplified `gain` times, which drives nodal densities and pressures negative
    (the input of the positivity limiter)."""
    U = random_state(cfg, seed)
    n = cfg.poly_deg + 1
    if cfg.dim == 2:
        q = U.reshape(-1, n * n, 4).copy()
        m = q.mean(axis=1, keepdims=True)
        q[::every] = m[::every] + gain * (q[::every] - m[::every])
    else:
        q = U.reshape(-1, 3, n).copy()
        m = q.mean(axis=2, keepdims=True)
        q[::every] = m[::every] + gain * (q[::every] - m[::every])
    return q.reshape(-1)
