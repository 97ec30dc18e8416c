"""ctypes wrapper of oracle/_ref/libfrsdg_ref.so: fr_sdg's own hot-path code
(include/*.hpp of the reference, compiled by oracle/ref_build.py against the
stand-ins of oracle/ref_shim) behind the same calls as oracle.Oracle.

TEST INFRASTRUCTURE ONLY: the tests use it to pin the restated oracle to the
reference, tests/golden/gen_ref_golden.py to freeze reference outputs as
fixtures, and bench.py's reference arm to time the reference's own residual on
the host cores.  The product package fr_sdg_b200 never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libfrsdg_ref.so"

_lib = None
_P, _D = C.c_void_p, C.c_double


def available() -> bool:
    """The library is built (from the reference tree when it is present)."""
    if LIB_PATH.exists():
        return True
    from oracle import ref_build

    return ref_build.build() is not None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} is not built and the reference tree is absent")
        L = C.CDLL(str(LIB_PATH))
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_create": (_P, [_P]),
            "ref_destroy": (None, [_P]),
            "ref_n_dofs": (C.c_int64, [_P]),
            "ref_set_threads": (None, [_P, C.c_int]),
            "ref_residual": (C.c_int, [_P, _D, _P, _P]),
            "ref_residual_complex": (C.c_int, [_P, _D, _P, _P]),
            "ref_rhs": (C.c_int, [_P, _D, _P, _P]),
            "ref_ifunction": (C.c_int, [_P, _D, _P, _P, _P]),
            "ref_jvp": (C.c_int, [_P, _D, _D, _P, _P, _P]),
            "ref_post_step": (C.c_int, [_P, _P]),
            "ref_prim_to_cons": (C.c_int, [_P, _P, _P]),
            "ref_reference_element": (C.c_int, [C.c_int, _D, _P, _P, _P, _P, _P]),
            "ref_filter_matrix": (C.c_int, [C.c_int, C.c_int, C.c_int, _D, _P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


def _chk(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().ref_last_error().decode()}")


class Reference:
    """The reference's residual path for one configuration (single rank)."""

    def __init__(self, cfg, threads: int = 1):
        self._h = lib().ref_create(C.addressof(cfg))
        if not self._h:
            raise RuntimeError(lib().ref_last_error().decode())
        self.n_dofs = int(lib().ref_n_dofs(self._h))
        if threads > 1:
            self.set_threads(threads)

    def set_threads(self, n: int) -> None:
        """2D residuals on n host threads, each owning a block of element rows as one
        MPI rank of the reference would (the ghost scatter and the residual of the
        block run on that thread)."""
        lib().ref_set_threads(self._h, n)

    def close(self):
        if self._h:
            lib().ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vec(self, a) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.n_dofs
        return a

    def residual(self, t: float, U) -> np.ndarray:
        U = self._vec(U)
        R = np.empty_like(U)
        _chk(lib().ref_residual(self._h, t, _p(U), _p(R)), "ref_residual")
        return R

    def residual_complex(self, t: float, U) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        R = np.empty_like(U)
        _chk(lib().ref_residual_complex(self._h, t, _p(U), _p(R)), "ref_residual_complex")
        return R

    def rhs(self, t: float, U, out: np.ndarray | None = None) -> np.ndarray:
        U = self._vec(U)
        F = np.empty_like(U) if out is None else out
        _chk(lib().ref_rhs(self._h, t, _p(U), _p(F)), "ref_rhs")
        return F

    def ifunction(self, t: float, U, Udot) -> np.ndarray:
        U, Udot = self._vec(U), self._vec(Udot)
        F = np.empty_like(U)
        _chk(lib().ref_ifunction(self._h, t, _p(U), _p(Udot), _p(F)), "ref_ifunction")
        return F

    def jvp(self, t: float, sigma: float, U, V) -> np.ndarray:
        U, V = self._vec(U), self._vec(V)
        JV = np.empty_like(U)
        _chk(lib().ref_jvp(self._h, t, sigma, _p(U), _p(V), _p(JV)), "ref_jvp")
        return JV

    def post_step(self, U) -> np.ndarray:
        U = self._vec(U).copy()
        _chk(lib().ref_post_step(self._h, _p(U)), "ref_post_step")
        return U

    def prim_to_cons(self, prim) -> np.ndarray:
        prim = self._vec(prim)
        out = np.empty_like(prim)
        _chk(lib().ref_prim_to_cons(self._h, _p(prim), _p(out)), "ref_prim_to_cons")
        return out


def default_config(c) -> None:
    """Fill a frsdg_config with the reference's defaults without the CUDA library:
    Parser::parse_options (parser.hpp:257-300: 10 elements, p = 3, box 1, c = 0),
    ConfigOptions and its option structs (parser.hpp:45-91: filter cut-off 2,
    strength 32, alpha 36, WENO gamma 0.998, shock theta 1, threshold 0.8, ideal gas
    gamma 1.4, R 287.05, VdW a 161.94, b 0.001265), outflow faces
    (boundary_conditions.hpp:229-235) and the complex step 1e-7
    (petsc_solver_impl.hpp:179)."""
    C.memset(C.addressof(c), 0, C.sizeof(c))
    c.dim, c.poly_deg = 2, 3
    c.n_elems[0] = c.n_elems[1] = 10
    c.box_length[0] = c.box_length[1] = 1.0
    c.radau_corr = 0.0
    c.gas_law, c.riemann = 0, 0
    c.gamma, c.R_spec, c.vdw_a, c.vdw_b = 1.4, 287.05, 161.94, 0.001265
    c.coord_sys = c.geometry = c.geom_profile = 0
    for f in range(4):
        c.bc[f].kind = 0
    c.apply_filter, c.filt_cut_off, c.filt_strength, c.filt_alpha = 0, 2, 32, 36.0
    c.apply_weno, c.weno_gamma, c.shock_theta, c.shock_threshold = 0, 0.998, 1.0, 0.8
    c.cond_sys, c.jvp_exact_bc, c.csd_eps = 0, 0, 1e-7
    # the positivity limiter has no counterpart in the reference: off, library floor
    c.pp_limit, c.pp_eps = 0, 1e-13


def reference_element(p: int, c: float = 0.0):
    n = p + 1
    x, w, dl, dr = (np.zeros(n) for _ in range(4))
    D = np.zeros((n, n))
    _chk(lib().ref_reference_element(p, c, _p(x), _p(w), _p(D), _p(dl), _p(dr)), "ref_reference_element")
    return x, w, D, dl, dr


def filter_matrix(p: int, cut_off: int = 2, strength: int = 32, alpha: float = 36.0) -> np.ndarray:
    n = p + 1
    F = np.zeros((n, n))
    _chk(lib().ref_filter_matrix(p, cut_off, strength, alpha, _p(F)), "ref_filter_matrix")
    return F
