"""Implicit time stepping over libfrsdg: backward Euler, inexact Newton, GMRES.

The reference hands implicit steps to PETSc (petsc_solver_impl.hpp:549-612):
TSBEULER calls the IFunction F(t, U, U_t) = U_t + R(M(U)) (fun_implicit, 626-655),
SNES newtonls solves F = 0 with a matrix-free Jacobian J = sigma dM/dU + dR/dU
applied by complex step (ComplexStepJacobianStrategy, 168-433), and KSP GMRES
solves each Newton system, preconditioned from a coloured Jacobian assembly.  This
module is the PETSc-free equivalent on the GPU:

  * J v       frsdg_jvp_prepare / frsdg_jvp (complex-step JVP kernel);
  * P^-1 r    frsdg_pc_setup / frsdg_pc_apply (element block-Jacobi: the diagonal
              blocks of J from one coloured complex-step launch, FP32 inverses), or
              frsdg_pc_setup_gs (red-black block Gauss-Seidel over all five blocks of an
              element row, from one distance-2 coloured launch);
  * GMRES(m)  right-preconditioned, classical Gram-Schmidt applied twice (the
              Arnoldi basis lives on the device; the small Hessenberg least-squares
              problem is solved on the host with Givens rotations, Saad, "Iterative
              Methods for Sparse Linear Systems", 2nd ed., section 6.5).

With a change of variables (cond_sys) the state is primitive and the transient
variable is M(U) = prim->cons (TSSetTransientVariable, 575): U_t is replaced by
(M(X) - M(U^n)) / dt.  Steady problems march in pseudo-time with the
switched-evolution-relaxation time step dt_k = dt_0 ||F_0|| / ||F_k|| (Mulder and
Van Leer, J. Comput. Phys. 59, 1985).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from ._abi import FrsdgError
from .solver import FRSolver


@dataclass
class GmresStats:
    iterations: int
    residual: float  # final preconditioned-system residual estimate, relative to ||b||


def gmres(matvec, precond, b: torch.Tensor, restart: int = 30, rtol: float = 1e-3, max_iter: int = 200) -> tuple[
        torch.Tensor, GmresStats]:
    """Solve A x = b, right-preconditioned: A M^-1 y = b, x = M^-1 y."""
    n = b.numel()
    x = torch.zeros_like(b)
    bnorm = float(torch.linalg.vector_norm(b))
    if bnorm == 0.0:
        return x, GmresStats(0, 0.0)
    V = torch.empty((restart + 1, n), dtype=b.dtype, device=b.device)
    Z = torch.empty((restart, n), dtype=b.dtype, device=b.device)
    w = torch.empty_like(b)
    total = 0
    rel = 1.0
    r = b.clone()
    while total < max_iter:
        beta = float(torch.linalg.vector_norm(r))
        rel = beta / bnorm
        if rel <= rtol:
            break
        V[0] = r / beta
        H = np.zeros((restart + 1, restart))
        cs = np.zeros(restart)
        sn = np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k = 0
        for j in range(restart):
            precond(V[j], Z[j])
            matvec(Z[j], w)
            h = V[: j + 1] @ w
            w -= V[: j + 1].T @ h
            h2 = V[: j + 1] @ w
            w -= V[: j + 1].T @ h2
            h = (h + h2).cpu().numpy()
            hn = float(torch.linalg.vector_norm(w))
            H[: j + 1, j] = h
            H[j + 1, j] = hn
            for i in range(j):
                t0 = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t0
            den = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if den == 0.0 else (H[j, j] / den, H[j + 1, j] / den)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            k = j + 1
            total += 1
            rel = abs(g[j + 1]) / bnorm
            if rel <= rtol or hn == 0.0 or total >= max_iter:
                break
            V[j + 1] = w / hn
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i]
        x += Z[:k].T @ torch.from_numpy(y).to(b.device)
        if rel <= rtol or total >= max_iter:
            break
        matvec(x, w)
        r = b - w
    return x, GmresStats(total, rel)


@dataclass
class NewtonStats:
    newton_iterations: int
    gmres_iterations: int
    f_norms: list = field(default_factory=list)


class BackwardEulerNewtonKrylov:
    """X^{n+1} solves F(t+dt, X, (M(X) - M(U^n))/dt) = 0 by inexact Newton with
    right-preconditioned GMRES; the Jacobian is sigma dM/dU + dR/dU, sigma = 1/dt."""

    def __init__(self, solver: FRSolver, restart: int = 30, gmres_rtol: float = 1e-3, max_gmres: int = 200,
                 newton_rtol: float = 1e-8, newton_atol: float = 1e-12, max_newton: int = 8,
                 precondition: bool | str = True):
        """precondition: True / "jacobi" (element block-Jacobi), "gs" (red-black block
        Gauss-Seidel over the five blocks of each element row) or False."""
        self.s = solver
        self.restart, self.gmres_rtol, self.max_gmres = restart, gmres_rtol, max_gmres
        self.newton_rtol, self.newton_atol, self.max_newton = newton_rtol, newton_atol, max_newton
        self.precondition = "jacobi" if precondition is True else precondition
        self.cond_sys = bool(solver.cfg.cond_sys)

    def _transient(self, X: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        if self.cond_sys:
            self.s.primitive_to_conservative(X, out)
        else:
            out.copy_(X)
        return out

    def step(self, U: torch.Tensor, t: float, dt: float) -> NewtonStats:
        """Advance U (in place) from t to t + dt."""
        s = self.s
        t1, sigma = t + dt, 1.0 / dt
        Mn = self._transient(U, torch.empty_like(U))
        MX = torch.empty_like(U)
        Xdot = torch.empty_like(U)
        F = torch.empty_like(U)
        stats = NewtonStats(0, 0)
        f0 = None
        for it in range(self.max_newton + 1):
            torch.sub(self._transient(U, MX), Mn, out=Xdot).mul_(sigma)
            s.fun_implicit(t1, U, Xdot, F)
            fn = float(torch.linalg.vector_norm(F))
            stats.f_norms.append(fn)
            if f0 is None:
                f0 = fn
            if fn <= max(self.newton_rtol * f0, self.newton_atol) or it == self.max_newton:
                break
            s.pre_jv_eval(t1, U, sigma)
            if self.precondition == "gs":
                s.pc_setup_gs(t1, sigma, U)
                precond = s.pc_apply
            elif self.precondition:
                s.pc_setup(t1, sigma, U)
                precond = s.pc_apply
            else:
                def precond(r, z):
                    z.copy_(r)
            dx, g = gmres(s.matmult, precond, -F, restart=self.restart, rtol=self.gmres_rtol,
                          max_iter=self.max_gmres)
            U += dx
            stats.newton_iterations += 1
            stats.gmres_iterations += g.iterations
        return stats


@dataclass
class SteadyStats:
    steps: int
    newton_iterations: int
    gmres_iterations: int
    residual_drop: float
    rejected: int = 0
    history: list = field(default_factory=list)


def march_to_steady(solver: FRSolver, U: torch.Tensor, dt0: float, drop: float = 1e-10, max_steps: int = 200,
                    dt_max: float = 1e6, newton: BackwardEulerNewtonKrylov | None = None,
                    max_rejections: int = 20, precondition: bool | str = True) -> SteadyStats:
    """Pseudo-transient continuation to a steady state: backward-Euler steps with the
    switched-evolution-relaxation time step until ||R(U)|| / ||R(U_0)|| <= drop.  A step
    that leaves a non-finite residual or a non-positive density (frsdg_status), or meets
    a singular element block in the preconditioner, is rejected and retried with a
    quarter of the time step, as a TS adaptor would."""
    nk = newton or BackwardEulerNewtonKrylov(solver, restart=60, max_gmres=400, max_newton=1, precondition=precondition)
    R = torch.empty_like(U)
    solver.residual_kernel(0.0, U, R)
    r0 = float(torch.linalg.vector_norm(R))
    solver.status()
    stats = SteadyStats(0, 0, 0, 1.0, 0, [1.0])
    U_prev = torch.empty_like(U)
    dt, t = dt0, 0.0
    while stats.steps < max_steps:
        U_prev.copy_(U)
        try:
            st = nk.step(U, t, dt)
        except FrsdgError:  # a singular element block at this state: reject the step
            st = None
        if st is not None:
            stats.newton_iterations += st.newton_iterations
            stats.gmres_iterations += st.gmres_iterations
            solver.residual_kernel(t + dt, U, R)
            rk = float(torch.linalg.vector_norm(R))
        if st is None or not math.isfinite(rk) or solver.status() != 0:
            stats.rejected += 1
            if stats.rejected > max_rejections:
                break
            U.copy_(U_prev)
            dt *= 0.25
            continue
        t += dt
        stats.steps += 1
        stats.residual_drop = rk / r0
        stats.history.append(stats.residual_drop)
        if stats.residual_drop <= drop:
            break
        dt = min(dt0 / stats.residual_drop, dt_max)
    return stats
