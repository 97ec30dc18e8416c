"""CPU: the positivity-preserving limiter of the oracle (Zhang and Shu, J. Comput. Phys.
229 (2010) 8918-8934; cfg.pp_limit, no counterpart in the reference) -- it keeps cell
averages, leaves admissible elements alone and makes every node admissible -- and, with
fr_sdg's own rhs and filter (oracle/_ref), keeps the circular explosion finite where
the reference's stabilisation alone does not."""
import numpy as np
import pytest

from fr_sdg_b200 import _abi as A
from oracle import oracle as O
from tests.cases import CASES_2D, _cfg2d, cfg1d
from tests.helpers import poisoned_state, random_state


def _pressure(cfg, rho, m2, E):
    e = (E - 0.5 * m2 / rho) / rho
    if cfg.gas_law == A.GAS_IDEAL:
        return (cfg.gamma - 1.0) * rho * e
    a, b = cfg.vdw_a, cfg.vdw_b
    return (cfg.gamma - 1.0) * rho * (e + a * rho) / (1.0 - b * rho) - a * rho * rho


def _nodes(cfg, U):
    """(rho, m2, E) per node and per-element quadrature weights."""
    n = cfg.poly_deg + 1
    w = O.reference_element(cfg.poly_deg)[1]
    if cfg.dim == 2:
        q = U.reshape(-1, n * n, 4)
        rho, m2, E = q[..., 0], q[..., 1] ** 2 + q[..., 2] ** 2, q[..., 3]
        W = np.outer(w, w).reshape(-1)
        return rho, m2, E, q, W
    q = U.reshape(-1, 3, n).transpose(0, 2, 1)
    return q[..., 0], q[..., 1] ** 2, q[..., 2], q, w


PP_CASES = {
    "cart_ideal": dict(name="cart_ideal_rusanov_p3"),
    "cart_vdw_p5": dict(name="cart_vdw_rusanov_p5_perx"),
    "sinewarp_p4": dict(name="sinewarp_hllc_p4_periodic"),
    "bump_p3": dict(name="bump_hllc_p3_inflow_outlet"),
}


def _cfg(case):
    return _cfg2d(**CASES_2D[PP_CASES[case]["name"]], pp_limit=True)


@pytest.mark.parametrize("case", sorted(PP_CASES))
def test_admissible_states_are_left_alone(case):
    cfg = _cfg(case)
    U = random_state(cfg, seed=5)
    assert np.array_equal(O.Oracle(cfg).pp_limit(U), U)


@pytest.mark.parametrize("case", sorted(PP_CASES))
def test_limited_state_is_admissible_and_keeps_cell_averages(case):
    cfg = _cfg(case)
    U = poisoned_state(cfg, seed=6)
    o = O.Oracle(cfg)
    L = o.pp_limit(U)
    rho0, _, _, _, _ = _nodes(cfg, U)
    assert (rho0 < 0).any() and not np.array_equal(L, U)
    rho, m2, E, q, W = _nodes(cfg, L)
    assert rho.min() > 0.0 and _pressure(cfg, rho, m2, E).min() > 0.0
    # cell averages with the quadrature weights of the limiter (detJ on curved meshes)
    if cfg.geometry in (A.GEOM_SINE_WARP, A.GEOM_WALL_PROFILE):
        J = o.node_metrics()[:, 4].reshape(-1, q.shape[1])
    else:
        J = np.ones(q.shape[:2])
    _, _, _, q0, _ = _nodes(cfg, U)
    Wj = W[None, :] * J
    mean0 = np.einsum("en,enc->ec", Wj, q0) / Wj.sum(axis=1)[:, None]
    mean1 = np.einsum("en,enc->ec", Wj, q) / Wj.sum(axis=1)[:, None]
    assert np.max(np.abs(mean1 - mean0)) <= 1e-13 * np.max(np.abs(mean0))
    # elements the poisoning did not touch are bit-identical
    per = q.shape[1] * q.shape[2]
    untouched = np.ones(len(q), bool)
    untouched[::3] = False
    assert np.array_equal(L.reshape(-1, per)[untouched], U.reshape(-1, per)[untouched])


@pytest.mark.parametrize("name", ["sod_rusanov_p3", "vdw_hllc_p5_walls", "p1_hllc_periodic"])
def test_limiter_1d(name):
    cfg = cfg1d(name, pp_limit=True)
    U = poisoned_state(cfg, seed=7)
    L = O.Oracle(cfg).pp_limit(U)
    rho, m2, E, q, w = _nodes(cfg, L)
    assert rho.min() > 0.0 and _pressure(cfg, rho, m2, E).min() > 0.0
    _, _, _, q0, _ = _nodes(cfg, U)
    assert np.allclose(np.einsum("n,enc->ec", w, q) / w.sum(), np.einsum("n,enc->ec", w, q0) / w.sum(),
                       rtol=0, atol=1e-13)


def test_post_step_applies_the_limiter_after_the_filter():
    """The filter alone turns a step profile negative (its top Legendre mode removed);
    with cfg.pp_limit the post-step ends admissible."""
    kw = dict(CASES_2D["cart_ideal_rusanov_p3"], apply_filter=True)
    cfg = _cfg2d(**kw)
    n = cfg.poly_deg + 1
    U = random_state(cfg, seed=8, amp=0.0).reshape(-1, n, n, 4)
    U[:, :, n // 2:, 0] *= 0.125  # density jump inside every element (x direction)
    U[:, :, n // 2:, 3] *= 0.1
    U = U.reshape(-1)
    plain = O.Oracle(cfg).post_step(U)
    assert plain.reshape(-1, 4)[:, 0].min() < 0.0
    cfg.pp_limit = 1
    lim = O.Oracle(cfg).post_step(U)
    q = lim.reshape(-1, 4)
    assert q[:, 0].min() > 0.0 and _pressure(cfg, q[:, 0], q[:, 1] ** 2 + q[:, 2] ** 2, q[:, 3]).min() > 0.0


def test_explosion_stays_finite_with_the_reference_rhs():
    """SSP-RK3 on the circular explosion (p = 4, filter on, CFL 0.1 with dt = CFL h /
    ((2p+1) c_max)): fr_sdg's own rhs and post-step (oracle/_ref) go negative within the
    first step; adding the oracle's positivity limiter on every stage keeps every node
    admissible to t = 0.05."""
    import torch

    from fr_sdg_b200.workloads import circular_explosion
    from oracle import reference

    if not reference.available():
        pytest.skip("oracle/_ref not built")
    wl = circular_explosion(12, 4, "ideal", 1.4, (0.0, 0.0), 0.4, 0.1)
    cfg = wl.cfg
    U = wl.init("cpu").numpy().copy()
    dt = wl.time_step(torch.from_numpy(U))
    r, o = reference.Reference(cfg), O.Oracle(cfg)

    def march(limit, steps):
        V = U.copy()
        for _ in range(steps):
            L = lambda X: r.rhs(0.0, X)
            V1 = limit(V + dt * L(V))
            V2 = limit(0.75 * V + 0.25 * (V1 + dt * L(V1)))
            V = limit(V / 3.0 + 2.0 / 3.0 * (V2 + dt * L(V2)))
            V = limit(r.post_step(V))
        return V

    bare = march(lambda X: X, 1).reshape(-1, 4)
    assert bare[:, 0].min() < 0.0  # the filter's overshoot
    steps = int(np.ceil(0.05 / dt))
    V = march(o.pp_limit, steps).reshape(-1, 4)
    assert np.all(np.isfinite(V)) and V[:, 0].min() > 0.0
    assert _pressure(cfg, V[:, 0], V[:, 1] ** 2 + V[:, 2] ** 2, V[:, 3]).min() > 0.0
