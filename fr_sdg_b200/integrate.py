"""Explicit time integration over the fused RK stages of libfrsdg.

The reference hands time stepping to PETSc TS (petsc_solver_impl.hpp:549-612):
SSP Runge-Kutta or classic RK4, the last step clipped to land on the final time
(TS_EXACTFINALTIME_MATCHSTEP, 556), and the post-step stabilisation after every
accepted step (604-607).  Here each stage is one frsdg_rk_stage call (residual
and update in one pass over the state):

  SSP-RK3 (Shu and Osher, J. Comput. Phys. 77, 1988):
    U1 = U + dt L(U);  U2 = 3/4 U + 1/4 U1 + dt/4 L(U1);  U+ = 1/3 U + 2/3 U2 + 2 dt/3 L(U2)
  RK4 (classic):  acc accumulates dt/6 (k1 + 2 k2 + 2 k3 + k4) on top of U.

Time step (cfl_time_step): dt = CFL * (L/N) / c_max(U0), c_max the largest
|velocity| + sound speed of the initial state (tools/run_test_matrix.py:40-52 take
c_max as an input), or with rule "dg" dt = CFL * (L/N) / ((2p + 1) c_max(U0)), the
(2p + 1)^-1 scaling of the explicit CFL ceilings that the reference's tools fit
(tools/c-vcjh_claude.py:410-430, tools/cfl_ceiling_plots.py:110-130).

With cfg.pp_limit the positivity limiter (frsdg_pp_limit) acts on every stage output
and the post-step applies it after the stabilisation, as the Zhang-Shu scheme needs
(J. Comput. Phys. 229 (2010) 8918-8934: SSP stages are convex combinations of Euler
steps, each of which the limiter keeps admissible).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import _abi as A
from .solver import FRSolver


def max_wave_speed(cfg: A.frsdg_config, U: torch.Tensor) -> float:
    """max(|v| + c) over the nodes, c from the configured gas law."""
    n = cfg.poly_deg + 1
    if cfg.dim == 2:
        q = U.view(-1, 4)
        rho, ru, rv, E = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    else:
        q = U.view(-1, 3, n)
        rho, ru, E = q[:, 0], q[:, 1], q[:, 2]
        rv = torch.zeros_like(rho)
    u, v = ru / rho, rv / rho
    e = E / rho - 0.5 * (u * u + v * v)
    g = cfg.gamma
    if cfg.gas_law == A.GAS_IDEAL:
        c2 = g * (g - 1.0) * e
    else:
        a, b = cfg.vdw_a, cfg.vdw_b
        cov = 1.0 - b * rho
        c2 = (g * (g - 1.0) * (e + a * rho)) / (cov * cov) + ((g - 1.0) * a * rho * (2.0 - b * rho)) / (cov * cov) \
            - 2.0 * a * rho
    return float((torch.sqrt(u * u + v * v) + torch.sqrt(c2)).max())


def cfl_time_step(cfg: A.frsdg_config, U0: torch.Tensor, cfl: float, rule: str = "h") -> float:
    """rule "h": CFL h / c_max; rule "dg": CFL h / ((2p + 1) c_max); h the smaller
    element size."""
    h = cfg.box_length[0] / cfg.n_elems[0]
    if cfg.dim == 2:
        h = min(h, cfg.box_length[1] / cfg.n_elems[1])
    if rule not in ("h", "dg"):
        raise ValueError("rule must be 'h' or 'dg'")
    scale = 1.0 if rule == "h" else 1.0 / (2 * cfg.poly_deg + 1)
    return cfl * scale * h / max_wave_speed(cfg, U0)


@dataclass
class RunStats:
    steps: int
    t: float
    dt: float
    rejected: int = 0  # steps rejected on the health word and retried as two half steps


class Integrator:
    """SSP-RK3 / RK4 over one FRSolver; buffers are allocated once.

    mixed=True: every stage takes the residual in FP32 arithmetic from its FP64 input,
    whose node primitives are recovered in FP64 (frsdg_rk_stage_mixed), and combines
    the stages in FP64; the FP64 state stays the solution."""

    def __init__(self, solver: FRSolver, scheme: str = "ssprk3", mixed: bool = False, before_stage=None):
        """before_stage(V): called with every stage input and with U before the post-step
        limiter -- a row-block partition refreshes its ghost rows there (FP64 stages)."""
        if scheme not in ("ssprk3", "rk4"):
            raise ValueError("scheme must be 'ssprk3' or 'rk4'")
        if mixed and (solver.cfg.dim != 2 or solver.cfg.cond_sys):
            raise ValueError("mixed precision: 2D configurations without change of variables")
        self.s = solver
        self.scheme = scheme
        self.mixed = mixed
        self.before = before_stage
        self._buf = None
        cfg = solver.cfg
        self.stabilise = bool(cfg.apply_filter or cfg.apply_weno)
        # the positivity limiter (cfg.pp_limit) acts on every stage output; the
        # post-step applies it again after the stabilisation
        self.pp = bool(cfg.pp_limit)
        # an element-local post-step (the filter overrides WENO when both are set) is
        # fused into the last stage of every step
        self.local_post = bool(cfg.apply_filter or not cfg.apply_weno) and (self.stabilise or self.pp)

    def _buffers(self, U: torch.Tensor):
        if self._buf is None or self._buf[0].device != U.device:
            self._buf = [torch.empty_like(U) for _ in range(3)]
        return self._buf

    def _rk(self, t: float, Us: torch.Tensor, out: torch.Tensor, post_step: bool = False, **kw) -> None:
        """One stage; the positivity limiter on its output and, with post_step, the whole
        post-step run in the stage's launch (frsdg_rk_stage_fused)."""
        if self.before is not None:
            self.before(Us)
        flags = (A.STAGE_MIXED if self.mixed else 0) | (A.STAGE_LIMIT if self.pp else 0)
        if post_step:
            flags |= A.STAGE_POST_STEP
        if flags:
            self.s.rk_stage_fused(t, Us, out, flags, **kw)
        else:
            self.s.rk_stage(t, Us, out, **kw)

    def step(self, U: torch.Tensor, t: float, dt: float) -> None:
        """Advance U (in place) from t to t + dt, then apply the post-step limiter.  An
        element-local post-step (the filter, the positivity limiter) runs inside the last
        stage's launch, which then writes U itself; the WENO limiter, which reads the
        neighbours, runs after it as its own pass."""
        s = self.s
        b1, b2, b3 = self._buffers(U)[:3]
        fuse = self.local_post  # the last stage writes U through the post-step
        separate = self.stabilise and not fuse
        if self.scheme == "ssprk3":
            last = b3 if separate else U
            self._rk(t, U, b1, gamma=dt, a=U, alpha=1.0)
            self._rk(t + dt, b1, b2, gamma=0.25 * dt, a=U, alpha=0.75, b=b1, beta=0.25)
            self._rk(t + 0.5 * dt, b2, last, post_step=fuse, gamma=2.0 * dt / 3.0, a=U, alpha=1.0 / 3.0, b=b2,
                     beta=2.0 / 3.0)
        else:
            last = b2 if separate else U
            b3.copy_(U)
            self._rk(t, U, b1, gamma=0.5 * dt, a=U, alpha=1.0, acc=b3, delta=dt / 6.0)
            self._rk(t + 0.5 * dt, b1, b2, gamma=0.5 * dt, a=U, alpha=1.0, acc=b3, delta=dt / 3.0)
            self._rk(t + 0.5 * dt, b2, b1, gamma=dt, a=U, alpha=1.0, acc=b3, delta=dt / 3.0)
            self._rk(t + dt, b1, last, post_step=fuse, gamma=dt / 6.0, a=b3, alpha=1.0)
        if separate:
            if self.before is not None:
                self.before(last)
            s.apply_stabilization_to(last, U)

    def time_dependent(self) -> bool:
        """Whether the residual reads t (the exact-vortex boundary kind)."""
        cfg = self.s.cfg
        faces = range(4) if cfg.dim == 2 else (A.LEFT, A.RIGHT)
        return any(cfg.bc[f].kind == A.BC_VORTEX for f in faces)

    def capture(self, U: torch.Tensor, dt: float, steps: int) -> torch.cuda.CUDAGraph:
        """`steps` full steps of size dt captured into one CUDA graph that updates U in
        place (kernel launches and device copies only: no allocation, no sync).  The
        capture runs on a side stream ordered after the current one."""
        scratch = U.clone()
        self.step(scratch, 0.0, dt)  # first calls set kernel attributes; buffers exist
        cur = torch.cuda.current_stream()
        side = torch.cuda.Stream(device=U.device)
        side.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            g.capture_begin()
            for _ in range(steps):
                self.step(U, 0.0, dt)
            g.capture_end()
        cur.wait_stream(side)
        return g

    def _guarded_step(self, U: torch.Tensor, t: float, dt: float, depth: int, max_reject: int) -> int:
        """One step with rejection (PETSc's -ts_max_reject, tools/c-vcjh_test.py:100-105):
        the step is taken from a saved copy of U; if the health word then reports a node
        with non-positive or non-finite density (in the stage inputs, read by the
        residuals, or in the result, read by frsdg_check_state), U is restored and the
        step is retried as two steps of dt/2, at most max_reject halvings deep.
        Returns the number of rejections."""
        while len(self._saved) <= depth:
            self._saved.append(torch.empty_like(U))
        saved = self._saved[depth]
        saved.copy_(U)
        self.s.status()  # clear the health word
        self.step(U, t, dt)
        self.s.check_state(U)
        if self.s.status() == 0:
            return 0
        if depth >= max_reject:
            raise RuntimeError(f"step at t = {t:.6g} failed after {max_reject} halvings of dt")
        U.copy_(saved)
        r = self._guarded_step(U, t, 0.5 * dt, depth + 1, max_reject)
        r += self._guarded_step(U, t + 0.5 * dt, 0.5 * dt, depth + 1, max_reject)
        return r + 1

    def run(self, U: torch.Tensor, dt: float, t_end: float | None = None, n_steps: int | None = None,
            t0: float = 0.0, graph: bool = False, steps_per_graph: int = 64, monitor=None,
            max_reject: int = 0) -> RunStats:
        """March to t_end (last step clipped to land on it) or for n_steps steps.  With
        graph=True (and a residual that does not read t) the full steps replay a CUDA
        graph of `steps_per_graph` steps; leftover and clipped steps run eagerly.
        monitor(step, t, U, final) is called with the initial state (step 0) and after
        every step (petsc_io.SolutionMonitor writes the PETSc solution file); a monitor
        that writes intermediate steps keeps the run eager.  max_reject > 0: every step
        checks the health word and a failed step is retried with halved steps
        (_guarded_step); such runs are eager and synchronise once per step."""
        if max_reject > 0:
            return self._run_guarded(U, dt, t_end, n_steps, t0, monitor, max_reject)
        tol = 1e-14 * max(1.0, abs(t_end)) if t_end is not None else 0.0
        if t_end is not None:
            n_full = 0
            while t0 + (n_full + 1) * dt <= t_end + tol:
                n_full += 1
        else:
            n_full = int(n_steps)
        t_acc = t0
        for _ in range(n_full):
            t_acc += dt
        n_total = n_full + (1 if t_end is not None and t_acc < t_end - tol else 0)
        if monitor is not None:
            monitor(0, t0, U, n_total == 0)
        t, k = t0, 0
        if graph and n_full >= steps_per_graph and not self.time_dependent() and self.before is None and (
                monitor is None or not monitor.every_step_matters):
            g = self.capture(U, dt, steps_per_graph)
            for _ in range(n_full // steps_per_graph):
                g.replay()
                for _ in range(steps_per_graph):
                    t += dt
                    k += 1
            del g
            if monitor is not None and k == n_total:
                monitor(k, t, U, True)
        while k < n_full:
            self.step(U, t, dt)
            t += dt
            k += 1
            if monitor is not None:
                monitor(k, t, U, k == n_total)
        if t_end is not None and t < t_end - tol:
            h = t_end - t
            self.step(U, t, h)
            t = t_end
            k += 1
            if monitor is not None:
                monitor(k, t, U, True)
        return RunStats(k, t, dt)

    def _run_guarded(self, U, dt, t_end, n_steps, t0, monitor, max_reject) -> RunStats:
        self._saved = []
        tol = 1e-14 * max(1.0, abs(t_end)) if t_end is not None else 0.0
        t, k, rej = t0, 0, 0
        if monitor is not None:
            monitor(0, t0, U, False)
        while (n_steps is None or k < n_steps) and (t_end is None or t < t_end - tol):
            h = dt if t_end is None else min(dt, t_end - t)
            rej += self._guarded_step(U, t, h, 0, max_reject)
            t = t + h if t_end is None or t + h < t_end - tol else t_end
            k += 1
            if monitor is not None:
                done = (n_steps is not None and k >= n_steps) or (t_end is not None and t >= t_end - tol)
                monitor(k, t, U, done)
        self._saved = []
        return RunStats(k, t, dt, rej)


def node_jacobian(cfg: A.frsdg_config, device="cpu") -> torch.Tensor:
    """detJ of the map (r, s) -> (x, y) at every node, [elem][l][k] flattened, for the
    Cartesian and sine-warped geometries (physics_evaluator.hpp:282-305)."""
    from .refelem import reference_element

    Nx, Ny, n = cfg.n_elems[0], cfg.n_elems[1], cfg.poly_deg + 1
    Lx, Ly = cfg.box_length[0], cfg.box_length[1]
    xr = torch.tensor(reference_element(cfg.poly_deg)[0], dtype=torch.float64, device=device)
    i = torch.arange(Nx, dtype=torch.float64, device=device)
    j = torch.arange(Ny, dtype=torch.float64, device=device)
    csi = (i[None, :, None, None] + 0.5 * (1 + xr[None, None, None, :])) / Nx
    eta = (j[:, None, None, None] + 0.5 * (1 + xr[None, None, :, None])) / Ny
    if cfg.geometry == A.GEOM_SINE_WARP:
        two_pi, amp = 2.0 * math.pi, cfg.geom_params[0]
        dc = two_pi * amp * torch.cos(two_pi * csi) * torch.sin(two_pi * eta)
        de = two_pi * amp * torch.sin(two_pi * csi) * torch.cos(two_pi * eta)
        det = (Lx + dc) * (Ly + de) - de * dc
    elif cfg.geometry == A.GEOM_CARTESIAN:
        det = torch.full_like(csi * eta, Lx * Ly)
    else:
        raise NotImplementedError("node_jacobian: Cartesian and sine-warp geometries only")
    det = det * (0.5 / Nx) * (0.5 / Ny)
    return det.expand(Ny, Nx, n, n).reshape(-1)


def l2_error(cfg: A.frsdg_config, U: torch.Tensor, exact: torch.Tensor, detJ: torch.Tensor | float = 1.0) -> torch.Tensor:
    """GLL-quadrature L2 error per conserved variable (compute_error,
    physics_impl_2D.hpp:203-265 / physics_impl_1D.hpp:245-324)."""
    from .refelem import reference_element

    n = cfg.poly_deg + 1
    w = torch.tensor(reference_element(cfg.poly_deg)[1], dtype=torch.float64, device=U.device)
    if cfg.dim == 2:
        d = (U - exact).view(-1, n, n, 4)
        wt = (w[:, None] * w[None, :])[None, :, :, None] * (detJ if isinstance(detJ, float) else detJ.view(-1, n, n, 1))
        return torch.sqrt((wt * d * d).sum(dim=(0, 1, 2)))
    d = (U - exact).view(-1, 3, n)
    jac = 0.5 * cfg.box_length[0] / cfg.n_elems[0]
    return torch.sqrt((w[None, None, :] * jac * d * d).sum(dim=(0, 2)))
