"""CPU: the host logic of the explicit integrator -- stage sequences, the clipped final
step and the solution-monitor schedule -- over a stand-in solver whose right-hand side
is rhs(U) = -U (so the exact solution is U0 exp(-t)) and whose limiter is the identity."""
from __future__ import annotations

import math
from types import SimpleNamespace

import pytest
import torch

from fr_sdg_b200 import _abi as A
from fr_sdg_b200.integrate import Integrator


class DecaySolver:
    """The rk_stage / apply_stabilization contract of FRSolver for dU/dt = -U."""

    def __init__(self, limiter: bool, pp: bool = False):
        self.cfg = SimpleNamespace(apply_filter=int(limiter), apply_weno=0, dim=2, cond_sys=0, pp_limit=int(pp),
                                   bc=[SimpleNamespace(kind=0) for _ in range(4)])
        self.stages = 0
        self.limits = 0
        self.pp_calls = []

    def rk_stage(self, t, Us, out, gamma, a=None, alpha=0.0, b=None, beta=0.0, acc=None, delta=0.0):
        assert out.data_ptr() != Us.data_ptr()
        v = -Us.clone()
        o = torch.zeros_like(Us)
        if a is not None:
            o = alpha * a
        if b is not None:
            o = o + beta * b
        if acc is not None:
            acc += delta * v
        out.copy_(o + gamma * v)
        self.stages += 1
        if gamma > self.unstable_above:
            self._bad += 1

    def rk_stage_fused(self, t, Us, out, flags, **kw):
        """frsdg_rk_stage_fused: the stage, then the post-step (filter) and the limiter."""
        self.rk_stage(t, Us, out, **kw)
        step = bool(flags & A.STAGE_POST_STEP)
        if step and (self.cfg.apply_filter or self.cfg.apply_weno):
            self.limits += 1
        if self.cfg.pp_limit and (step or flags & A.STAGE_LIMIT):
            self.pp_calls.append(out.data_ptr())

    def apply_stabilization(self, U):
        self.limits += 1

    def pp_limit(self, U, U32=None):
        self.pp_calls.append(U.data_ptr())

    # health word: a stage with gamma above `unstable_above` "goes bad"
    unstable_above = float("inf")
    _bad = 0

    def check_state(self, U):
        pass

    def status(self):
        b, self._bad = self._bad, 0
        return b

    def apply_stabilization_to(self, src, dst):
        assert src.data_ptr() != dst.data_ptr()
        dst.copy_(src)
        self.limits += 1


@pytest.mark.parametrize("scheme,order", [("ssprk3", 3), ("rk4", 4)])
@pytest.mark.parametrize("limiter", [False, True])
def test_stage_sequences_converge_at_their_order(scheme, order, limiter):
    errs = []
    for n in (20, 40):
        s = DecaySolver(limiter)
        U = torch.ones(8, dtype=torch.float64)
        st = Integrator(s, scheme).run(U, 1.0 / n, t_end=1.0)
        assert st.steps == n and abs(st.t - 1.0) < 1e-14
        assert s.stages == n * (3 if scheme == "ssprk3" else 4)
        assert s.limits == (n if limiter else 0)
        errs.append(float((U - math.exp(-1.0)).abs().max()))
    rate = math.log2(errs[0] / errs[1])
    assert abs(rate - order) < 0.2, (errs, rate)


@pytest.mark.parametrize("scheme", ["ssprk3", "rk4"])
def test_positivity_limiter_acts_on_every_stage_output(scheme):
    """cfg.pp_limit: the limiter runs on the output of every stage (Zhang-Shu needs
    each Euler sub-step admissible), the last stage's output included."""
    s = DecaySolver(limiter=True, pp=True)
    U = torch.ones(8, dtype=torch.float64)
    it = Integrator(s, scheme)
    it.step(U, 0.0, 0.1)
    assert len(s.pp_calls) == s.stages == (3 if scheme == "ssprk3" else 4)
    assert s.limits == 1
    s2 = DecaySolver(limiter=False, pp=False)
    Integrator(s2, scheme).step(torch.ones(8, dtype=torch.float64), 0.0, 0.1)
    assert s2.pp_calls == []


def test_step_rejection_halves_failed_steps():
    """max_reject: a step whose health word reports bad nodes is undone and retaken as two
    half steps (PETSc's -ts_max_reject); the result is the one of the half steps."""
    s = DecaySolver(limiter=False)
    s.unstable_above = 0.06  # the first SSP-RK3 stage has gamma = dt
    U = torch.ones(4, dtype=torch.float64)
    st = Integrator(s, "ssprk3").run(U, 0.1, t_end=1.0, max_reject=3)
    assert st.steps == 10 and st.rejected == 10 and abs(st.t - 1.0) < 1e-14
    g = lambda h: 1 - h + h * h / 2 - h ** 3 / 6
    assert abs(float(U[0]) - g(0.05) ** 20) < 1e-14
    # two levels: dt = 0.2 fails, 0.1 fails, 0.05 passes
    s2 = DecaySolver(limiter=False)
    s2.unstable_above = 0.06
    U2 = torch.ones(4, dtype=torch.float64)
    st2 = Integrator(s2, "ssprk3").run(U2, 0.2, t_end=0.4, max_reject=3)
    assert st2.steps == 2 and st2.rejected == 2 * 3 and abs(float(U2[0]) - g(0.05) ** 8) < 1e-14
    # a step that no halving rescues
    s3 = DecaySolver(limiter=False)
    s3.unstable_above = 0.001
    with pytest.raises(RuntimeError):
        Integrator(s3, "ssprk3").run(torch.ones(4, dtype=torch.float64), 0.1, n_steps=2, max_reject=2)


def test_clipped_final_step_and_monitor_schedule():
    """t_end = 10.5 dt: ten full steps and one clipped step of dt/2; a monitor with
    interval 4 sees steps 0, 4, 8 and the final step 11."""
    s = DecaySolver(limiter=True)
    U = torch.ones(4, dtype=torch.float64)
    dt = 0.05
    seen = []

    class Monitor:
        every_step_matters = True

        def __call__(self, step, t, V, final):
            if step % 4 == 0 or final:
                seen.append((step, round(t / dt, 9), final))

    st = Integrator(s, "ssprk3").run(U, dt, t_end=10.5 * dt, monitor=Monitor())
    assert st.steps == 11 and abs(st.t - 10.5 * dt) < 1e-15
    assert seen == [(0, 0.0, False), (4, 4.0, False), (8, 8.0, False), (11, 10.5, True)]
    # the clipped step is the exact SSP-RK3 map with h = dt / 2 after ten full steps
    g = lambda h: 1 - h + h * h / 2 - h ** 3 / 6
    assert abs(float(U[0]) - g(dt) ** 10 * g(dt / 2)) < 1e-15


def test_before_stage_hook_sees_every_stage_input_and_the_limiter_input():
    """The ghost-row hook runs before every stage and, when the post-step reads the
    neighbours (WENO alone), before it; an element-local post-step (the filter) is part
    of the last stage's launch and needs no refresh."""
    s = DecaySolver(limiter=True)
    s.cfg.apply_filter, s.cfg.apply_weno = 0, 1
    U = torch.ones(4, dtype=torch.float64)
    calls = []
    Integrator(s, "ssprk3", before_stage=lambda V: calls.append(V.data_ptr())).step(U, 0.0, 0.1)
    assert len(calls) == 4 and calls[0] == U.data_ptr() and calls[3] != U.data_ptr()
    assert s.limits == 1
    s = DecaySolver(limiter=True)
    calls = []
    Integrator(s, "ssprk3", before_stage=lambda V: calls.append(V.data_ptr())).step(U, 0.0, 0.1)
    assert len(calls) == 3 and calls[0] == U.data_ptr()
    assert s.limits == 1


def test_cfl_time_step_uniform_states():
    """dt = CFL (L/N) / max(|v| + c): ideal gas c^2 = gamma p / rho; Van der Waals
    c^2 = [gamma (gamma-1)(e + a rho) + (gamma-1) a rho (2 - b rho)] / (1 - b rho)^2 - 2 a rho
    (gas_models.hpp:89-158), from the state's specific internal energy."""
    from fr_sdg_b200.integrate import cfl_time_step
    from fr_sdg_b200.workloads import make_config, pack2d, rhoE

    n_nodes = 3 * 2 * 16
    rho, u, v, p, g = 1.2, 0.3, -0.4, 0.9, 1.4
    for gas, (a, b) in (("ideal", (0.0, 0.0)), ("vdw", (0.05, 0.02))):
        # element sizes 0.2 (x) and 0.1 (y): the time step takes the smaller one
        cfg = make_config(dim=2, p=3, n_elems=(3, 2), box=(0.6, 0.2), gas=gas, vdw=(a, b))
        ones = torch.ones(n_nodes, dtype=torch.float64)
        E = rhoE(gas, g, a, b, rho * ones, (u * u + v * v) * ones, p * ones)
        U = pack2d(rho * ones, rho * u * ones, rho * v * ones, E)
        dt = cfl_time_step(cfg, U, 0.5)
        if gas == "ideal":
            c = math.sqrt(g * p / rho)
        else:
            e = float(E[0]) / rho - 0.5 * (u * u + v * v)
            cov = 1.0 - b * rho
            c = math.sqrt((g * (g - 1) * (e + a * rho) + (g - 1) * a * rho * (2 - b * rho)) / (cov * cov) - 2 * a * rho)
            # the state's pressure from the same gas law
            assert abs((g - 1) * rho * (e + a * rho) / cov - a * rho * rho - p) < 1e-12
        assert abs(dt - 0.5 * 0.1 / (math.hypot(u, v) + c)) < 1e-12 * dt, gas
        # the "dg" rule divides by 2p + 1
        assert abs(cfl_time_step(cfg, U, 0.5, "dg") - dt / 7.0) < 1e-12 * dt, gas
