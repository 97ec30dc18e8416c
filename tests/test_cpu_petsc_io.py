"""PETSc binary solution files: the reader restated from the reference's tools, the
record sizes of the library and the monitor's step schedule (no GPU needed)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fr_sdg_b200 import _abi as A
from fr_sdg_b200.petsc_io import SolutionMonitor
from oracle.petsc_binary import VEC_FILE_CLASSID, last_vector, read_all_vectors, record_bytes


def _vectors(seed=5):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(n) for n in (0, 1, 7, 1000)]


@pytest.mark.parametrize("index_bytes", [4, 8])
def test_reader_reads_appended_records(tmp_path, index_bytes):
    """read_all_vectors (tools/plot.py:109-129) reads records of either header width."""
    vs = _vectors()
    f = tmp_path / "sol.bin"
    f.write_bytes(b"".join(record_bytes(v, index_bytes) for v in vs))
    got = read_all_vectors(f)
    assert len(got) == len(vs)
    for a, b in zip(got, vs):
        assert a.dtype == np.dtype(">f8") and np.array_equal(a.astype(np.float64), b)


def test_record_layout_and_last_vector(tmp_path):
    """Header = big-endian class id 1211214 and length; tools/check_iso_vortex.py keeps
    the last complete record and skips a truncated one."""
    x = np.array([1.0, -2.5, np.inf])
    rec = record_bytes(x)
    assert rec[:8] == bytes([0x00, 0x12, 0x7B, 0x4E, 0, 0, 0, 3])
    assert int.from_bytes(rec[:4], "big") == VEC_FILE_CLASSID
    assert rec[8:16] == bytes([0x3F, 0xF0, 0, 0, 0, 0, 0, 0])  # 1.0, most significant byte first
    f = tmp_path / "sol.bin"
    y = np.arange(4.0)
    f.write_bytes(rec + record_bytes(y) + record_bytes(np.ones(5))[:-8])
    assert np.array_equal(last_vector(f), y)


def test_library_record_sizes():
    lib = A.lib()
    nb = C.c_int64()
    assert lib.frsdg_petsc_vec_record_bytes(10, 4, C.byref(nb)) == 0 and nb.value == 88
    assert lib.frsdg_petsc_vec_record_bytes(10, 8, C.byref(nb)) == 0 and nb.value == 96
    assert lib.frsdg_petsc_vec_record_bytes(0, 4, C.byref(nb)) == 0 and nb.value == 8
    assert lib.frsdg_petsc_vec_record_bytes(2 ** 31, 8, C.byref(nb)) == 0 and nb.value == 16 + 8 * 2 ** 31
    assert lib.frsdg_petsc_vec_record_bytes(2 ** 31, 4, C.byref(nb)) == A.ERR_ARG
    assert lib.frsdg_petsc_vec_record_bytes(10, 2, C.byref(nb)) == A.ERR_ARG
    assert lib.frsdg_petsc_vec_record_bytes(-1, 4, C.byref(nb)) == A.ERR_ARG


@pytest.mark.parametrize("interval,skip,expect", [
    (1, False, [0, 1, 2, 3, 4, 5, 6, 7]),
    (3, False, [0, 3, 6, 7]),
    (3, True, [3, 6, 7]),
    (-1, False, [7]),
    (-1, True, [7]),
])
def test_monitor_schedule(tmp_path, interval, skip, expect):
    """Step k is written when k % interval == 0 and at the final step (7 here); step 0
    is the initial state, left out by skip_initial; interval -1: final state only."""
    with SolutionMonitor(tmp_path / "s.bin", interval=interval, skip_initial=skip) as m:
        got = [k for k in range(8) if m.wants(k, k == 7)]
    assert got == expect
    with pytest.raises(ValueError):
        SolutionMonitor(tmp_path / "t.bin", interval=0)
