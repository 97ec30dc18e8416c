"""fr_sdg_b200: B200 implementation of fr_sdg's Flux Reconstruction residual path.

The compute lives in libfrsdg.so (C ABI: include/frsdg.h); this package is the
host mirror of the reference's PETSc callback surface over it.
"""
from . import _abi
from ._abi import FrsdgError, frsdg_bc, frsdg_config, lib
from .refelem import filter_matrix, reference_element
from .solver import FRSolver

__all__ = ["FRSolver", "FrsdgError", "frsdg_bc", "frsdg_config", "lib", "reference_element",
           "filter_matrix", "_abi"]
