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
  * coarse    optional second level (CoarseCorrection): the Galerkin operator
              P^T J P on piecewise-constant aggregates of elements, probed with 20
              JVPs (aggregates coloured (I + 2J) mod 5, four variables), inverted
              densely; applied before the element-block sweep;
  * GMRES(m)  right-preconditioned; every Arnoldi step (classical Gram-Schmidt with
              the DGKS second pass, the Hessenberg column and its Givens rotations,
              Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., section
              6.5) runs in libfrsdg's kernels (frsdg_gmres_arnoldi); the host reads one
              residual norm per step, two steps late, and one per restart cycle.

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

from . import _abi as A
from ._abi import FrsdgError
from .solver import FRSolver, _stream


@dataclass
class GmresStats:
    iterations: int
    residual: float  # final preconditioned-system residual estimate, relative to ||b||


class _DeviceArnoldi:
    """The Arnoldi step and the back substitution of GMRES(m) in libfrsdg
    (frsdg_gmres_arnoldi, frsdg_gmres_solve): Gram-Schmidt with the DGKS second pass,
    the Hessenberg column and its Givens rotations stay on the device."""

    def __init__(self, n: int, device):
        self.lib = A.lib()
        self.n = n
        self.work = torch.empty(int(self.lib.frsdg_gmres_work_doubles(n)), dtype=torch.float64, device=device)

    def arnoldi(self, V, j, w, H, cs, sn, g, inv):
        A.check(self.lib.frsdg_gmres_arnoldi(V.data_ptr(), V.stride(0), j, w.data_ptr(), self.n, H.data_ptr(),
                                             H.stride(0), cs.data_ptr(), sn.data_ptr(), g.data_ptr(), inv.data_ptr(),
                                             self.work.data_ptr(), _stream()), "frsdg_gmres_arnoldi")

    def solve(self, H, g, k, y):
        A.check(self.lib.frsdg_gmres_solve(H.data_ptr(), H.stride(0), g.data_ptr(), k, y.data_ptr(), _stream()),
                "frsdg_gmres_solve")


class _HostArnoldi:
    """The same step in torch operations on host tensors: the CPU form of the driver's
    numerics, for tests of the restart and convergence logic without a GPU."""

    def arnoldi(self, V, j, w, H, cs, sn, g, inv):
        Vj = V[: j + 1]
        w0 = float(w @ w)
        h = Vj @ w
        w -= Vj.T @ h
        w1 = float(w @ w)
        if w1 < 0.5 * w0:  # DGKS: a second pass
            h2 = Vj @ w
            w -= Vj.T @ h2
            h = h + h2
            w1 = float(w @ w)
        hn = math.sqrt(max(w1, 0.0))
        H[: j + 1, j] = h
        H[j + 1, j] = hn
        for i in range(j):
            a, b_ = float(H[i, j]), float(H[i + 1, j])
            H[i, j] = cs[i] * a + sn[i] * b_
            H[i + 1, j] = -sn[i] * a + cs[i] * b_
        a, b_ = float(H[j, j]), float(H[j + 1, j])
        den = math.hypot(a, b_)
        c, s_ = (1.0, 0.0) if den == 0.0 else (a / den, b_ / den)
        cs[j], sn[j] = c, s_
        H[j, j] = c * a + s_ * b_
        H[j + 1, j] = 0.0
        gj = float(g[j])
        g[j + 1] = -s_ * gj
        g[j] = c * gj
        inv[0] = 1.0 / hn if hn > 0.0 else 0.0

    def solve(self, H, g, k, y):
        for i in range(k - 1, -1, -1):
            d = float(H[i, i])
            y[i] = (float(g[i]) - float(H[i, i + 1:k] @ y[i + 1:k])) / d if d != 0.0 else 0.0


class _LaggedNorm:
    """|g[idx]| read back `lag` Arnoldi steps late: each step queues a copy of its new
    residual norm into pinned host memory and waits only for the copy of `lag` steps ago,
    so the host stays at most `lag` steps ahead of the GPU and the GPU never waits for
    the host.  lag = 0 reads at once (host tensors)."""

    def __init__(self, g: torch.Tensor, lag: int):
        self.g, self.lag = g, lag
        if lag:
            self.buf = torch.empty(lag + 1, dtype=g.dtype, pin_memory=True)
            self.ev = [torch.cuda.Event() for _ in range(lag + 1)]
        self.count = 0

    def reset(self) -> None:
        self.count = 0

    def push(self, idx: int) -> float | None:
        if not self.lag:
            return abs(float(self.g[idx]))
        slot = self.count % (self.lag + 1)
        self.buf[slot: slot + 1].copy_(self.g[idx: idx + 1], non_blocking=True)
        self.ev[slot].record()
        self.count += 1
        if self.count <= self.lag:
            return None
        old = (self.count - 1 - self.lag) % (self.lag + 1)
        self.ev[old].synchronize()
        return abs(float(self.buf[old]))


def gmres(matvec, precond, b: torch.Tensor, restart: int = 30, rtol: float = 1e-3, max_iter: int = 200,
          lag: int = 2) -> tuple[torch.Tensor, GmresStats]:
    """Solve A x = b, right-preconditioned: A M^-1 y = b, x = M^-1 y (GMRES(restart),
    Saad, algorithm 6.9).  On CUDA tensors every Arnoldi step runs in libfrsdg's kernels
    and the host reads one residual norm per step, `lag` steps late (the solve may take
    up to `lag` extra steps past the tolerance; each cycle's true estimate is read once
    at its end).  At most 256 steps per cycle."""
    if restart > 256:
        raise ValueError("gmres: at most 256 Arnoldi steps per cycle")
    n = b.numel()
    x = torch.zeros_like(b)
    bnorm = float(torch.linalg.vector_norm(b))
    if bnorm == 0.0:
        return x, GmresStats(0, 0.0)
    dev = b.device
    f64 = dict(dtype=torch.float64, device=dev)
    V = torch.empty((restart + 1, n), dtype=b.dtype, device=dev)
    Z = torch.empty((restart, n), dtype=b.dtype, device=dev)
    w = torch.empty_like(b)
    H = torch.zeros((restart + 1, restart), **f64)
    cs, sn, y = torch.zeros(restart, **f64), torch.zeros(restart, **f64), torch.zeros(restart, **f64)
    g = torch.zeros(restart + 1, **f64)
    inv = torch.zeros(1, **f64)
    step = _DeviceArnoldi(n, dev) if b.is_cuda else _HostArnoldi()
    probe = _LaggedNorm(g, lag if b.is_cuda else 0)
    total = 0
    rel = 1.0
    r = b.clone()
    while total < max_iter:
        beta = float(torch.linalg.vector_norm(r))
        rel = beta / bnorm
        if rel <= rtol:
            break
        torch.div(r, beta, out=V[0])
        H.zero_()
        g.zero_()
        g[0] = beta
        probe.reset()
        k = 0
        for j in range(restart):
            precond(V[j], Z[j])
            matvec(Z[j], w)
            step.arnoldi(V, j, w, H, cs, sn, g, inv)
            torch.mul(w, inv, out=V[j + 1])
            k = j + 1
            total += 1
            seen = probe.push(j + 1)
            if (seen is not None and seen <= rtol * bnorm) or total >= max_iter:
                break
        step.solve(H, g, k, y)
        x.addmv_(Z[:k].T, y[:k])
        rel = abs(float(g[k])) / bnorm
        if rel <= rtol or total >= max_iter:
            break
        matvec(x, w)
        r = b - w
    return x, GmresStats(total, rel)


class CoarseCorrection:
    """Second level of the preconditioner: z = P A_c^-1 P^T r with P the injection of
    one constant state per aggregate of ax x ay elements (per variable) and
    A_c = P^T J P the Galerkin coarse operator.

    J couples an element to its face neighbours only, so J P couples an aggregate to
    its four face-neighbour aggregates: colouring the aggregates by (I + 2J) mod 5
    gives every closed five-aggregate neighbourhood distinct colours, and A_c follows
    from 5 colours x 4 variables = 20 JVPs (the way the element blocks are probed by
    frsdg_jac_blocks5).  A_c (4 * aggregates square, FP64) is inverted (or LU-factorised)
    once per set-up; meshes of a few thousand aggregates keep it small."""

    def __init__(self, cfg: A.frsdg_config, ax: int = 4, ay: int = 4, explicit_inverse: bool = True):
        """explicit_inverse: keep A_c^-1, applied as one dense matrix-vector product
        (0.02 ms for 4,096 unknowns on a B200, against 1.0 ms for the two triangular
        solves of its LU factors; the inverse costs 25 ms instead of 16 ms once per
        Newton step), or keep the LU factors."""
        if cfg.dim != 2:
            raise ValueError("coarse correction: 2D meshes only")
        for f in range(4):
            if cfg.bc[f].kind == A.BC_PERIODIC:  # (I + 2J) mod 5 would need counts divisible by 5
                raise ValueError("coarse correction: non-periodic meshes only")
        self.nx, self.ny = cfg.n_elems[0], cfg.n_elems[1]
        n = cfg.poly_deg + 1
        self.nn = n * n
        self.ax, self.ay = ax, ay
        self.gx, self.gy = -(-self.nx // ax), -(-self.ny // ay)
        self.nagg = self.gx * self.gy
        self.nc = 4 * self.nagg
        self.explicit_inverse = explicit_inverse
        self._lu = None
        self._inv = None
        self._dev = None

    def _maps(self, device):
        if self._dev != device:
            i = torch.arange(self.nx, device=device)
            j = torch.arange(self.ny, device=device)
            I, J = (i // self.ax)[None, :], (j // self.ay)[:, None]
            self.elem_agg = (J * self.gx + I).reshape(-1)            # aggregate of each element
            gi = torch.arange(self.gx, device=device)[None, :]
            gj = torch.arange(self.gy, device=device)[:, None]
            self.colour = ((gi + 2 * gj) % 5).reshape(-1)             # colour of each aggregate
            self._dev = device
        return self.elem_agg

    def restrict(self, r: torch.Tensor) -> torch.Tensor:
        """P^T r: per aggregate and variable, the sum over its elements' nodes (plain
        reductions in a fixed order, so repeated calls give identical bits)."""
        per_elem = r.view(self.ny, self.nx, self.nn, 4).sum(2)
        py, px = self.gy * self.ay - self.ny, self.gx * self.ax - self.nx
        if px or py:
            per_elem = torch.nn.functional.pad(per_elem, (0, 0, 0, px, 0, py))
        return per_elem.view(self.gy, self.ay, self.gx, self.ax, 4).sum((1, 3)).reshape(self.nagg, 4)

    def prolong(self, zc: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """out = P zc: every node of an aggregate takes the aggregate's state."""
        ea = self._maps(out.device)
        out.view(-1, self.nn, 4).copy_(zc.view(self.nagg, 4)[ea].unsqueeze(1).expand(-1, self.nn, 4))
        return out

    def neighbour_of_colour(self, c: int, device) -> torch.Tensor:
        """For every aggregate, the aggregate of colour c in its closed face
        neighbourhood (itself, right, top, bottom, left), or -1 when there is none."""
        self._maps(device)
        k = torch.arange(self.nagg, device=device)
        I, J = k % self.gx, k // self.gx
        d = (c - self.colour) % 5  # colour offsets: +1 right, -1 left, +2 top, -2 bottom
        di = torch.where(d == 1, 1, torch.where(d == 4, -1, 0))
        dj = torch.where(d == 2, 1, torch.where(d == 3, -1, 0))
        I2, J2 = I + di, J + dj
        ok = (I2 >= 0) & (I2 < self.gx) & (J2 >= 0) & (J2 < self.gy)
        return torch.where(ok, J2 * self.gx + I2, torch.full_like(k, -1))

    def assemble(self, matvec, template: torch.Tensor) -> torch.Tensor:
        """A_c = P^T J P by coloured probing: 20 JVPs."""
        dev = template.device
        self._maps(dev)
        A = torch.zeros(self.nagg, 4, self.nagg, 4, dtype=torch.float64, device=dev)
        e = torch.empty_like(template)
        w = torch.empty_like(template)
        rows = torch.arange(self.nagg, device=dev)
        for c in range(5):
            src = self.neighbour_of_colour(c, dev)
            has = src >= 0
            sel = (self.colour == c).to(template.dtype)
            for v in range(4):
                zc = torch.zeros(self.nagg, 4, dtype=template.dtype, device=dev)
                zc[:, v] = sel
                matvec(self.prolong(zc, e), w)
                rw = self.restrict(w)
                A[rows[has], :, src[has], v] = rw[has]
        return A.view(self.nc, self.nc)

    def setup(self, matvec, template: torch.Tensor) -> None:
        A_c = self.assemble(matvec, template)
        if self.explicit_inverse:
            self._inv = torch.linalg.inv(A_c)
        else:
            self._lu = torch.linalg.lu_factor(A_c)

    def solve(self, r: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """out = P A_c^-1 P^T r."""
        rc = self.restrict(r).reshape(self.nc, 1)
        zc = self._inv @ rc if self.explicit_inverse else torch.linalg.lu_solve(*self._lu, rc)
        return self.prolong(zc, out)


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
                 precondition: bool | str = True, coarse: tuple[int, int] | None = None):
        """precondition: True / "jacobi" (element block-Jacobi), "gs" (red-black block
        Gauss-Seidel over the five blocks of each element row) or False.
        coarse=(ax, ay): add the aggregate coarse level (CoarseCorrection) in front of
        the element-block preconditioner: z = zc + M^-1 (r - J zc), zc = P A_c^-1 P^T r."""
        self.s = solver
        self.restart, self.gmres_rtol, self.max_gmres = restart, gmres_rtol, max_gmres
        self.newton_rtol, self.newton_atol, self.max_newton = newton_rtol, newton_atol, max_newton
        self.precondition = "jacobi" if precondition is True else precondition
        self.cond_sys = bool(solver.cfg.cond_sys)
        if coarse and solver.n_dofs != solver.n_dofs_global:
            raise ValueError("coarse correction: whole meshes only (no row window)")
        self.coarse = CoarseCorrection(solver.cfg, *coarse) if coarse else None
        self._w = None

    def _two_level(self, smoother):
        cc, s = self.coarse, self.s

        def apply(r, z):
            if self._w is None or self._w[0].shape != r.shape:
                self._w = (torch.empty_like(r), torch.empty_like(r))
            zc, w = self._w
            cc.solve(r, zc)
            s.matmult(zc, w)
            torch.sub(r, w, out=w)
            smoother(w, z)
            z += zc
        return apply

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
            if self.coarse is not None:
                self.coarse.setup(s.matmult, U)
                precond = self._two_level(precond)
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
                    max_rejections: int = 20, precondition: bool | str = True,
                    max_growth: float | None = None, stall: float | None = None,
                    reject_growth: float | None = None) -> SteadyStats:
    """Pseudo-transient continuation to a steady state: backward-Euler steps with the
    switched-evolution-relaxation time step until ||R(U)|| / ||R(U_0)|| <= drop.  A step
    that leaves a non-finite residual or a non-positive density (frsdg_status), or meets
    a singular element block in the preconditioner, is rejected and retried with a
    quarter of the time step, as a TS adaptor would.  max_growth caps the ratio of
    consecutive time steps; with stall, a step that leaves the residual above stall
    times the previous one halves the time step instead of the SER update; with
    reject_growth, a step that multiplies the residual by more than that is rejected."""
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
        rk = math.nan
        if st is not None:
            stats.newton_iterations += st.newton_iterations
            stats.gmres_iterations += st.gmres_iterations
            solver.residual_kernel(t + dt, U, R)
            rk = float(torch.linalg.vector_norm(R))
        bad = solver.status()  # read (and clear) the health word after every attempt
        grew = reject_growth is not None and rk > reject_growth * stats.history[-1] * r0
        if st is None or not math.isfinite(rk) or bad != 0 or grew:
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
        prev = stats.history[-2]
        if stall is not None and stats.residual_drop > stall * prev:
            dt = 0.5 * dt
            continue
        dt_new = min(dt0 / stats.residual_drop, dt_max)
        dt = dt_new if max_growth is None else min(dt_new, max_growth * dt)
    return stats
