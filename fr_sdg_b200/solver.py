"""FRSolver: the reference's PETSc callback surface over libfrsdg.

Method names follow PetscSolver and ComplexStepJacobianStrategy
(include/petsc_solver_impl.hpp): rhs_func (657-670), fun_implicit (626-655),
pre_jv_eval (223-248), matmult (250-267), apply_stabilization (683-702) and
primitive_to_conservative (719-727), plus residual_kernel
(physics_impl_2D.hpp:646-902).  Vectors are torch float64 CUDA tensors in the
DMDA natural layout; every call is ordered on torch's current CUDA stream.
Errors raise FrsdgError with the library's message, like PetscCall.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi as A


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class FRSolver:
    def __init__(self, cfg: A.frsdg_config):
        self.cfg = cfg
        self._lib = A.lib()
        h = C.c_void_p()
        A.check(self._lib.frsdg_create(C.byref(cfg), C.byref(h)), "frsdg_create")
        self._h = h
        n = C.c_int64()
        A.check(self._lib.frsdg_n_dofs(h, C.byref(n)), "frsdg_n_dofs")
        self.n_dofs = int(n.value)
        self.n_elems = cfg.n_elems[0] * (cfg.n_elems[1] if cfg.dim == 2 else 1)
        self.n_dofs_global = self.n_dofs

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if self._h:
            self._lib.frsdg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check_vec(self, *vs: torch.Tensor) -> None:
        for v in vs:
            if v.dtype != torch.float64 or not v.is_cuda or not v.is_contiguous() or v.numel() != self.n_dofs:
                raise ValueError(f"expected a contiguous float64 CUDA vector of {self.n_dofs} entries")

    def set_row_window(self, row_base: int, rows: int, row_begin: int, row_end: int) -> None:
        """Work on a row block of the mesh (frsdg_set_row_window): vectors then hold
        `rows` element rows from global row `row_base`, of which [row_begin, row_end)
        are computed; rows = 0 restores the whole mesh."""
        A.check(self._lib.frsdg_set_row_window(self._h, row_base, rows, row_begin, row_end), "frsdg_set_row_window")
        cfg = self.cfg
        nx = cfg.n_elems[0]
        nd = self.n_dofs_global // (nx * cfg.n_elems[1])
        self.n_elems = nx * (rows if rows else cfg.n_elems[1])
        self.n_dofs = self.n_elems * nd

    # -- PETSc callbacks --------------------------------------------------
    def residual_kernel(self, t: float, U: torch.Tensor, R: torch.Tensor) -> None:
        self._check_vec(U, R)
        A.check(self._lib.frsdg_residual(self._h, t, _ptr(U), _ptr(R), _stream()), "frsdg_residual")

    def rhs_func(self, t: float, U: torch.Tensor, rhs: torch.Tensor) -> None:
        self._check_vec(U, rhs)
        A.check(self._lib.frsdg_rhs(self._h, t, _ptr(U), _ptr(rhs), _stream()), "frsdg_rhs")

    def fun_implicit(self, t: float, U: torch.Tensor, U_t: torch.Tensor, F: torch.Tensor) -> None:
        self._check_vec(U, U_t, F)
        A.check(self._lib.frsdg_ifunction(self._h, t, _ptr(U), _ptr(U_t), _ptr(F), _stream()), "frsdg_ifunction")

    def rk_stage(self, t: float, Us: torch.Tensor, out: torch.Tensor, gamma: float,
                 a: torch.Tensor | None = None, alpha: float = 0.0, b: torch.Tensor | None = None,
                 beta: float = 0.0, acc: torch.Tensor | None = None, delta: float = 0.0) -> None:
        """out = alpha a + beta b + gamma rhs(Us); acc += delta rhs(Us) -- one fused RK stage."""
        self._check_vec(Us, out, *(v for v in (a, b, acc) if v is not None))
        p = lambda v: _ptr(v) if v is not None else None
        A.check(self._lib.frsdg_rk_stage(self._h, t, _ptr(Us), p(a), alpha, p(b), beta, gamma, _ptr(out),
                                         p(acc), delta, _stream()), "frsdg_rk_stage")

    def rk_stage_fused(self, t: float, Us: torch.Tensor, out: torch.Tensor, flags: int, gamma: float,
                       a: torch.Tensor | None = None, alpha: float = 0.0, b: torch.Tensor | None = None,
                       beta: float = 0.0, acc: torch.Tensor | None = None, delta: float = 0.0) -> None:
        """rk_stage with the element-local work after it in the same launch (flags: A.STAGE_*):
        the mixed residual, the positivity limiter on out, or the whole post-step on out."""
        self._check_vec(Us, out, *(v for v in (a, b, acc) if v is not None))
        p = lambda v: _ptr(v) if v is not None else None
        A.check(self._lib.frsdg_rk_stage_fused(self._h, t, _ptr(Us), p(a), alpha, p(b), beta, gamma, _ptr(out),
                                               p(acc), delta, int(flags), _stream()), "frsdg_rk_stage_fused")

    def _check_f32(self, *vs: torch.Tensor) -> None:
        for v in vs:
            if v.dtype != torch.float32 or not v.is_cuda or not v.is_contiguous() or v.numel() != self.n_dofs:
                raise ValueError(f"expected a contiguous float32 CUDA vector of {self.n_dofs} entries")

    def residual_kernel_f32(self, t: float, U32: torch.Tensor, R32: torch.Tensor) -> None:
        """The residual in FP32 from an FP32 state (mixed-precision form)."""
        self._check_f32(U32, R32)
        A.check(self._lib.frsdg_residual_f32(self._h, t, _ptr(U32), _ptr(R32), _stream()), "frsdg_residual_f32")

    def rk_stage_mixed(self, t: float, Us: torch.Tensor, out: torch.Tensor, gamma: float,
                       a: torch.Tensor | None = None, alpha: float = 0.0, b: torch.Tensor | None = None,
                       beta: float = 0.0, acc: torch.Tensor | None = None, delta: float = 0.0) -> None:
        """out = alpha a + beta b + gamma rhs32(Us) in FP64, acc += delta rhs: the residual
        in FP32 arithmetic from the FP64 state Us, node primitives recovered in FP64."""
        self._check_vec(Us, out, *(v for v in (a, b, acc) if v is not None))
        p = lambda v: _ptr(v) if v is not None else None
        A.check(self._lib.frsdg_rk_stage_mixed(self._h, t, _ptr(Us), p(a), alpha, p(b), beta, gamma, _ptr(out),
                                               p(acc), delta, _stream()), "frsdg_rk_stage_mixed")

    def pre_jv_eval(self, t: float, U: torch.Tensor, sigma: float) -> None:
        self._check_vec(U)
        self._jvp_U = U  # keep alive while the library holds the pointer
        A.check(self._lib.frsdg_jvp_prepare(self._h, t, sigma, _ptr(U)), "frsdg_jvp_prepare")

    def matmult(self, v: torch.Tensor, out: torch.Tensor) -> None:
        self._check_vec(v, out)
        A.check(self._lib.frsdg_jvp(self._h, _ptr(v), _ptr(out), _stream()), "frsdg_jvp")

    def jac_blocks(self, t: float, sigma: float, U: torch.Tensor, blocks: torch.Tensor) -> None:
        """Element-diagonal Jacobian blocks (coloured complex step), blocks[e] column-major."""
        self._check_vec(U)
        nd = self.n_dofs // self.n_elems
        if blocks.dtype != torch.float64 or not blocks.is_cuda or not blocks.is_contiguous() \
                or blocks.numel() != self.n_elems * nd * nd:
            raise ValueError(f"expected a contiguous float64 CUDA tensor of {self.n_elems * nd * nd} entries")
        A.check(self._lib.frsdg_jac_blocks(self._h, t, sigma, _ptr(U), _ptr(blocks), _stream()), "frsdg_jac_blocks")

    def pc_setup(self, t: float, sigma: float, U: torch.Tensor) -> None:
        """Block-Jacobi preconditioner at (t, sigma, U): blocks and their FP32 inverses."""
        self._check_vec(U)
        A.check(self._lib.frsdg_pc_setup(self._h, t, sigma, _ptr(U), _stream()), "frsdg_pc_setup")

    def jac_blocks5(self, t: float, sigma: float, U: torch.Tensor, blocks5: torch.Tensor) -> None:
        """All five blocks of every element row (distance-2 coloured complex step)."""
        self._check_vec(U)
        nd = self.n_dofs // self.n_elems
        if blocks5.dtype != torch.float64 or not blocks5.is_cuda or not blocks5.is_contiguous() \
                or blocks5.numel() != 5 * self.n_elems * nd * nd:
            raise ValueError(f"expected a contiguous float64 CUDA tensor of {5 * self.n_elems * nd * nd} entries")
        A.check(self._lib.frsdg_jac_blocks5(self._h, t, sigma, _ptr(U), _ptr(blocks5), _stream()), "frsdg_jac_blocks5")

    def pc_setup_gs(self, t: float, sigma: float, U: torch.Tensor) -> None:
        """Red-black block Gauss-Seidel preconditioner at (t, sigma, U)."""
        self._check_vec(U)
        A.check(self._lib.frsdg_pc_setup_gs(self._h, t, sigma, _ptr(U), _stream()), "frsdg_pc_setup_gs")

    def pc_apply(self, r: torch.Tensor, z: torch.Tensor) -> None:
        """z = inv(block diagonal) r."""
        self._check_vec(r, z)
        A.check(self._lib.frsdg_pc_apply(self._h, _ptr(r), _ptr(z), _stream()), "frsdg_pc_apply")

    def apply_stabilization(self, U: torch.Tensor) -> None:
        self._check_vec(U)
        A.check(self._lib.frsdg_post_step(self._h, _ptr(U), _stream()), "frsdg_post_step")

    def apply_stabilization_to(self, src: torch.Tensor, dst: torch.Tensor) -> None:
        """dst = limit(src) without touching src (no counterpart in the reference)."""
        self._check_vec(src, dst)
        A.check(self._lib.frsdg_post_step_to(self._h, _ptr(src), _ptr(dst), _stream()), "frsdg_post_step_to")

    def pp_limit(self, U: torch.Tensor, U32: torch.Tensor | None = None) -> None:
        """Positivity limiter on U in place (cfg.pp_limit; no counterpart in the
        reference); U32, an FP32 copy of U, is refreshed where U changes."""
        self._check_vec(U)
        if U32 is not None:
            self._check_f32(U32)
        A.check(self._lib.frsdg_pp_limit(self._h, _ptr(U), _ptr(U32) if U32 is not None else None, _stream()),
                "frsdg_pp_limit")

    def primitive_to_conservative(self, inp: torch.Tensor, out: torch.Tensor) -> None:
        self._check_vec(inp, out)
        A.check(self._lib.frsdg_prim_to_cons(self._h, _ptr(inp), _ptr(out), _stream()), "frsdg_prim_to_cons")

    def rhs_func_host(self, t: float, U_host: torch.Tensor, rhs_host: torch.Tensor) -> None:
        """rhs_func on host (ideally pinned) float64 tensors; returns when done."""
        for v in (U_host, rhs_host):
            if v.dtype != torch.float64 or v.is_cuda or not v.is_contiguous() or v.numel() != self.n_dofs:
                raise ValueError("expected contiguous float64 host vectors")
        A.check(self._lib.frsdg_rhs_host(self._h, t, _ptr(U_host), _ptr(rhs_host), _stream()), "frsdg_rhs_host")

    def check_state(self, U: torch.Tensor) -> None:
        """Count the nodes of U with non-positive or non-finite density into the health
        word (read by status())."""
        self._check_vec(U)
        A.check(self._lib.frsdg_check_state(self._h, _ptr(U), _stream()), "frsdg_check_state")

    def status(self) -> int:
        """Nodes with non-positive or non-finite density seen since the last call."""
        n = C.c_int64()
        A.check(self._lib.frsdg_status(self._h, C.byref(n)), "frsdg_status")
        return int(n.value)
