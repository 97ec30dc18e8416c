"""GPU: full explicit runs through the fused RK stages against the same
integrator driven by the oracle on the CPU, plus physical checks (exact vortex,
exact Riemann solution of the Sod tube)."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200.integrate import Integrator, cfl_time_step, l2_error, node_jacobian
from fr_sdg_b200.workloads import blast_large, exact_vortex, node_coords, pack2d, sod1d, vortex_curved
from oracle.oracle import Oracle
from tests.helpers import rel_err
from fr_sdg_b200.exact_riemann import sod_exact

pytestmark = pytest.mark.gpu


def oracle_run(cfg, U0: np.ndarray, dt: float, n_steps: int, scheme: str) -> np.ndarray:
    """The integrator of fr_sdg_b200.integrate with the oracle's rhs and post-step."""
    o = Oracle(cfg, threads=4)
    stab = bool(cfg.apply_filter or cfg.apply_weno)

    def stage(t, Us, gamma, a=None, alpha=0.0, b=None, beta=0.0, acc=None, delta=0.0):
        v = o.rhs(t, Us)
        out = np.zeros_like(Us)
        if a is not None:
            out = alpha * a
        if b is not None:
            out = out + beta * b
        out = out + gamma * v
        if acc is not None:
            acc += delta * v
        return o.pp_limit(out) if cfg.pp_limit else out

    U, t = U0.copy(), 0.0
    for _ in range(n_steps):
        if scheme == "ssprk3":
            U1 = stage(t, U, dt, a=U, alpha=1.0)
            U2 = stage(t + dt, U1, 0.25 * dt, a=U, alpha=0.75, b=U1, beta=0.25)
            U = stage(t + 0.5 * dt, U2, 2.0 * dt / 3.0, a=U, alpha=1.0 / 3.0, b=U2, beta=2.0 / 3.0)
        else:
            acc = U.copy()
            U1 = stage(t, U, 0.5 * dt, a=U, alpha=1.0, acc=acc, delta=dt / 6.0)
            U2 = stage(t + 0.5 * dt, U1, 0.5 * dt, a=U, alpha=1.0, acc=acc, delta=dt / 3.0)
            U3 = stage(t + 0.5 * dt, U2, dt, a=U, alpha=1.0, acc=acc, delta=dt / 3.0)
            U = stage(t + dt, U3, dt / 6.0, a=acc, alpha=1.0)
        if stab:
            U = o.post_step(U)
        t += dt
    return U


@pytest.mark.parametrize("name", ["sod1d", "vortex_rk4", "blast_vdw"])
def test_run_matches_oracle_integrator(name, cuda):
    if name == "sod1d":
        wl, steps = sod1d(), 30
    elif name == "vortex_rk4":
        wl, steps = vortex_curved(n_elems=12, p=4), 10
    else:
        wl, steps = blast_large(n_elems=16, p=5), 10
    U0 = wl.init("cpu").numpy()
    dt = wl.time_step(torch.from_numpy(U0))
    scheme = "rk4" if wl.integrator == "rk4" else "ssprk3"
    ref = oracle_run(wl.cfg, U0, dt, steps, scheme)
    with FRSolver(wl.cfg) as s:
        U = torch.from_numpy(U0).to(cuda)
        Integrator(s, scheme).run(U, dt, n_steps=steps)
        got = U.cpu().numpy()
    err = rel_err(got, ref)
    assert err <= 1e-11, f"{name}: rel err {err:.3e} after {steps} steps"


def test_vortex_converges_to_exact(cuda):
    """Isentropic vortex on the sine-warped periodic mesh: L2 density error against
    the exact translated vortex falls with resolution (p = 4, t = 1)."""
    errs = []
    for ne in (16, 32):
        wl = vortex_curved(n_elems=ne, p=4)
        with FRSolver(wl.cfg) as s:
            U = wl.init(cuda)
            dt = cfl_time_step(wl.cfg, U, 0.05)
            Integrator(s, "rk4").run(U, dt, t_end=1.0)
            x, y = node_coords(wl.cfg, cuda)
            ex = pack2d(*exact_vortex(1.0, x, y))
            errs.append(float(l2_error(wl.cfg, U, ex, node_jacobian(wl.cfg, cuda))[0]))
            assert s.status() == 0
    assert errs[1] < errs[0] / 8.0, f"L2 density errors {errs}"
    assert errs[1] < 2e-3


def test_sod_against_exact_riemann(cuda):
    """1D Sod tube (N = 200, p = 3, Rusanov, spectral filter + positivity limiter, SSP-RK3,
    CFL 0.1) at t = 0.2 against the exact Riemann solution: L1 density error small."""
    wl = sod1d()
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        dt = wl.time_step(U)
        st = Integrator(s, "ssprk3").run(U, dt, t_end=wl.t_end)
        assert abs(st.t - 0.2) < 1e-12
        x, _ = node_coords(wl.cfg, "cpu")
    rho = U.view(-1, 3, 4)[:, 0].cpu().numpy()
    rho_ex = sod_exact(x.numpy(), 0.2)
    w = np.array([1 / 6, 5 / 6, 5 / 6, 1 / 6]) * 0.5 * (1.0 / 200)
    l1 = float(np.sum(w[None, :] * np.abs(rho - rho_ex)))
    assert l1 < 5e-3, f"L1 density error {l1:.3e}"


@pytest.mark.parametrize("name", ["vortex_rk4", "sod1d_weno"])
def test_graph_replay_matches_eager(name, cuda):
    """The CUDA-graph replay of full steps gives the eager run's state bit for bit."""
    if name == "vortex_rk4":
        wl, scheme = vortex_curved(n_elems=12, p=4), "rk4"
    else:
        wl, scheme = sod1d(), "ssprk3"
    with FRSolver(wl.cfg) as s:
        U0 = wl.init(cuda)
        dt = wl.time_step(U0)
        Ue, Ug = U0.clone(), U0.clone()
        t_end = 25.5 * dt
        se = Integrator(s, scheme).run(Ue, dt, t_end=t_end)
        sg = Integrator(s, scheme).run(Ug, dt, t_end=t_end, graph=True, steps_per_graph=8)
        assert se.steps == sg.steps == 26 and abs(sg.t - t_end) < 1e-15 and sg.t == se.t
        assert torch.equal(Ue, Ug)
        assert s.status() == 0
