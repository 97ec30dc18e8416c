"""ctypes wrapper of the CPU oracle (oracle/build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker of the CUDA library.  The product
package fr_sdg_b200 never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "liboracle.so"

_lib = None
_P, _D = C.c_void_p, C.c_double


def build() -> Path:
    """Compile the oracle with make (a few seconds)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        sig = {
            "oracle_last_error": (C.c_char_p, []),
            "oracle_create": (_P, [_P]),
            "oracle_destroy": (None, [_P]),
            "oracle_set_threads": (None, [_P, C.c_int]),
            "oracle_n_dofs": (C.c_int64, [_P]),
            "oracle_residual": (C.c_int, [_P, _D, _P, _P]),
            "oracle_residual_complex": (C.c_int, [_P, _D, _P, _P]),
            "oracle_rhs": (C.c_int, [_P, _D, _P, _P]),
            "oracle_ifunction": (C.c_int, [_P, _D, _P, _P, _P]),
            "oracle_jvp": (C.c_int, [_P, _D, _D, _P, _P, _P]),
            "oracle_post_step": (C.c_int, [_P, _P]),
            "oracle_pp_limit": (C.c_int, [_P, _P]),
            "oracle_prim_to_cons": (C.c_int, [_P, _P, _P]),
            "oracle_reference_element": (C.c_int, [C.c_int, _D, _P, _P, _P, _P, _P]),
            "oracle_filter_matrix": (C.c_int, [C.c_int, C.c_int, C.c_int, _D, _P]),
            "oracle_node_metrics": (C.c_int, [_P, _P]),
            "oracle_node_coords": (C.c_int, [_P, _P]),
            "oracle_count_flops": (C.c_int, [_P, _D, _P, _P]),
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
        raise RuntimeError(f"{what}: {lib().oracle_last_error().decode()}")


class Oracle:
    """CPU restatement of the reference residual path for one configuration."""

    def __init__(self, cfg, threads: int = 1):
        self._h = lib().oracle_create(C.addressof(cfg))
        if not self._h:
            raise RuntimeError(lib().oracle_last_error().decode())
        lib().oracle_set_threads(self._h, threads)
        self.n_dofs = int(lib().oracle_n_dofs(self._h))

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n: int) -> None:
        lib().oracle_set_threads(self._h, n)

    def _vec(self, a) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.n_dofs
        return a

    def residual(self, t: float, U) -> np.ndarray:
        U = self._vec(U)
        R = np.empty_like(U)
        _chk(lib().oracle_residual(self._h, t, _p(U), _p(R)), "oracle_residual")
        return R

    def residual_complex(self, t: float, U: np.ndarray) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        R = np.empty_like(U)
        _chk(lib().oracle_residual_complex(self._h, t, _p(U), _p(R)), "oracle_residual_complex")
        return R

    def rhs(self, t: float, U) -> np.ndarray:
        U = self._vec(U)
        F = np.empty_like(U)
        _chk(lib().oracle_rhs(self._h, t, _p(U), _p(F)), "oracle_rhs")
        return F

    def ifunction(self, t: float, U, Udot) -> np.ndarray:
        U, Udot = self._vec(U), self._vec(Udot)
        F = np.empty_like(U)
        _chk(lib().oracle_ifunction(self._h, t, _p(U), _p(Udot), _p(F)), "oracle_ifunction")
        return F

    def jvp(self, t: float, sigma: float, U, V) -> np.ndarray:
        U, V = self._vec(U), self._vec(V)
        JV = np.empty_like(U)
        _chk(lib().oracle_jvp(self._h, t, sigma, _p(U), _p(V), _p(JV)), "oracle_jvp")
        return JV

    def post_step(self, U) -> np.ndarray:
        U = self._vec(U).copy()
        _chk(lib().oracle_post_step(self._h, _p(U)), "oracle_post_step")
        return U

    def pp_limit(self, U) -> np.ndarray:
        """The positivity limiter (cfg.pp_limit's stage limiter) applied to a copy of U."""
        U = self._vec(U).copy()
        _chk(lib().oracle_pp_limit(self._h, _p(U)), "oracle_pp_limit")
        return U

    def prim_to_cons(self, prim) -> np.ndarray:
        prim = self._vec(prim)
        out = np.empty_like(prim)
        _chk(lib().oracle_prim_to_cons(self._h, _p(prim), _p(out)), "oracle_prim_to_cons")
        return out

    def count_flops(self, t: float, U) -> dict:
        """Arithmetic of one residual evaluation, counted by the counting scalar of
        flop_count.cpp: additions, multiplications, divisions, square roots, exp/log/pow."""
        U = self._vec(U)
        c = np.zeros(5, dtype=np.uint64)
        _chk(lib().oracle_count_flops(self._h, t, _p(U), c.ctypes.data), "oracle_count_flops")
        return dict(zip(("add", "mul", "div", "sqrt", "other"), (int(v) for v in c)))

    def node_metrics(self) -> np.ndarray:
        out = np.empty(self.n_dofs // 4 * 5)
        _chk(lib().oracle_node_metrics(self._h, _p(out)), "oracle_node_metrics")
        return out.reshape(-1, 5)

    def node_coords(self) -> np.ndarray:
        out = np.empty(self.n_dofs // 4 * 2)
        _chk(lib().oracle_node_coords(self._h, _p(out)), "oracle_node_coords")
        return out.reshape(-1, 2)


def reference_element(p: int, c: float = 0.0):
    n = p + 1
    x, w, dl, dr = (np.zeros(n) for _ in range(4))
    D = np.zeros((n, n))
    _chk(lib().oracle_reference_element(p, c, _p(x), _p(w), _p(D), _p(dl), _p(dr)), "oracle_reference_element")
    return x, w, D, dl, dr


def filter_matrix(p: int, cut_off: int = 2, strength: int = 32, alpha: float = 36.0) -> np.ndarray:
    n = p + 1
    F = np.zeros((n, n))
    _chk(lib().oracle_filter_matrix(p, cut_off, strength, alpha, _p(F)), "oracle_filter_matrix")
    return F
