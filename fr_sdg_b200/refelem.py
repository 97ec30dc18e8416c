"""Host-side reference element and filter matrix from libfrsdg (no GPU needed)."""
from __future__ import annotations

import ctypes as C
from functools import lru_cache

import numpy as np

from . import _abi as A


@lru_cache(maxsize=None)
def reference_element(p: int, radau_corr: float = 0.0):
    """(nodes, weights, D, dL, dR) of degree p: GLL (reference_element.hpp:50-147) and
    CachedElementData (cached_computations.hpp:8-137) as built by the library."""
    n = p + 1
    x, w, dl, dr = (np.zeros(n) for _ in range(4))
    D = np.zeros((n, n))
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    A.check(A.lib().frsdg_reference_element(p, radau_corr, ptr(x), ptr(w), ptr(D), ptr(dl), ptr(dr)),
            "frsdg_reference_element")
    for a in (x, w, D, dl, dr):
        a.setflags(write=False)
    return x, w, D, dl, dr


def filter_matrix(p: int, cut_off: int = 2, strength: int = 32, alpha: float = 36.0) -> np.ndarray:
    """V diag(sigma) V^-1 (filter.hpp:451-484) as built by the library."""
    n = p + 1
    F = np.zeros((n, n))
    A.check(A.lib().frsdg_filter_matrix(p, cut_off, strength, alpha, F.ctypes.data_as(C.c_void_p)),
            "frsdg_filter_matrix")
    return F
