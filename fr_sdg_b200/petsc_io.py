"""Solution files in PETSc's binary Vec format, as `-ts_monitor_solution` writes them.

The reference writes its solutions through PETSc's solution monitor, configured on
the command line (TSSetFromOptions, petsc_solver_impl.hpp:557):

    -ts_monitor_solution binary:<file>
    -ts_monitor_solution_interval <k>     (-1: the final state only)
    -ts_monitor_solution_skip_initial

and its tools read the file record by record (tools/plot.py:109-129,
tools/check_iso_vortex.py:215-233).  SolutionMonitor writes the same bytes for the
PETSc-free integrator, so those tools read GPU results unchanged: each record is
packed on the device by frsdg_petsc_vec_pack (class id, length, big-endian
doubles), copied once into pinned host memory and appended to the file.

Which steps are written follows PETSc's TSMonitorSolution rule: step k when
k % interval == 0 (interval > 0), and the final step for any non-zero interval;
step 0 is the initial state, left out by skip_initial.  PETSc is not available to
run here, so this schedule restates its documented option semantics.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from . import _abi as A


def pack_record(x: torch.Tensor, index_bytes: int = 4, out: torch.Tensor | None = None) -> torch.Tensor:
    """The PETSc binary record of the FP64 CUDA vector x as a uint8 CUDA tensor
    (packed on torch's current stream)."""
    if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
        raise ValueError("x must be a contiguous float64 CUDA tensor")
    lib = A.lib()
    nb = C.c_int64()
    A.check(lib.frsdg_petsc_vec_record_bytes(x.numel(), index_bytes, C.byref(nb)), "frsdg_petsc_vec_record_bytes")
    if out is None or out.numel() != nb.value or out.device != x.device:
        out = torch.empty(nb.value, dtype=torch.uint8, device=x.device)
    A.check(lib.frsdg_petsc_vec_pack(x.data_ptr(), x.numel(), index_bytes, out.data_ptr(),
                                     torch.cuda.current_stream(x.device).cuda_stream), "frsdg_petsc_vec_pack")
    return out


class SolutionMonitor:
    """`-ts_monitor_solution binary:<path>` for Integrator.run(monitor=...)."""

    def __init__(self, path: str | os.PathLike, interval: int = 1, skip_initial: bool = False,
                 index_bytes: int = 4, append: bool = False):
        if interval == 0 or interval < -1:
            raise ValueError("interval must be positive or -1 (final state only)")
        self.path = os.fspath(path)
        self.interval = int(interval)
        self.skip_initial = bool(skip_initial)
        self.index_bytes = int(index_bytes)
        self.records = 0
        self._dev = None
        self._host = None
        self._f = open(self.path, "ab" if append else "wb")

    def wants(self, step: int, final: bool) -> bool:
        if step == 0 and self.skip_initial:
            return False
        return (self.interval > 0 and step % self.interval == 0) or final

    @property
    def every_step_matters(self) -> bool:
        """Whether steps other than the last may be written (a replayed CUDA graph
        of many steps cannot stop in between)."""
        return self.interval > 0

    def __call__(self, step: int, t: float, U: torch.Tensor, final: bool = False) -> bool:
        if not self.wants(step, final):
            return False
        self.write(U)
        return True

    def write(self, U: torch.Tensor) -> None:
        self._dev = pack_record(U.reshape(-1), self.index_bytes, self._dev)
        if self._host is None or self._host.numel() != self._dev.numel():
            self._host = torch.empty(self._dev.numel(), dtype=torch.uint8, pin_memory=True)
        self._host.copy_(self._dev)  # synchronous: the bytes are complete on return
        self._f.write(memoryview(self._host.numpy()))
        self.records += 1

    def close(self) -> None:
        if self._f is not None:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
