"""Reader of PETSc binary Vec files, as the reference's post-processing tools read them.

TEST INFRASTRUCTURE ONLY: the checker of the library's PETSc record writer
(frsdg_petsc_vec_pack, fr_sdg_b200.petsc_io).  Nothing in fr_sdg_b200 imports it.

Restates two readers of the reference:
  read_all_vectors   tools/plot.py:109-129 -- records appended one after the other;
                     a big-endian int32 pair (class id, length) and, when the class
                     id is not 1211214, the pair re-read as big-endian int64 (PETSc
                     with 64-bit indices); then `length` big-endian doubles.
  last_vector        tools/check_iso_vortex.py:215-233 -- int32 headers only, the
                     class id must be 1211214, the last complete record wins.
"""
from __future__ import annotations

import numpy as np

VEC_FILE_CLASSID = 1211214


def read_all_vectors(path) -> list[np.ndarray]:
    vectors = []
    with open(path, "rb") as f:
        while True:
            header = np.fromfile(f, dtype=">i4", count=2)
            if header.size == 0:
                break
            classid, size = int(header[0]), int(header[1])
            if classid != VEC_FILE_CLASSID:
                f.seek(-8, 1)
                header = np.fromfile(f, dtype=">i8", count=2)
                classid, size = int(header[0]), int(header[1])
            vectors.append(np.fromfile(f, dtype=">f8", count=size))
    return vectors


def last_vector(path) -> np.ndarray:
    last = None
    with open(path, "rb") as f:
        while True:
            header = np.fromfile(f, dtype=">i4", count=2)
            if len(header) < 2:
                break
            if int(header[0]) != VEC_FILE_CLASSID:
                raise ValueError("not a PETSc Vec record")
            data = np.fromfile(f, dtype=">f8", count=int(header[1]))
            if len(data) == int(header[1]):
                last = data
    if last is None:
        raise ValueError(f"{path}: no complete record")
    return last


def record_bytes(x: np.ndarray, index_bytes: int = 4) -> bytes:
    """The record a PETSc binary viewer writes for the FP64 vector x (numpy's own
    big-endian encoding), for comparing against the device packer byte for byte."""
    it = ">i4" if index_bytes == 4 else ">i8"
    head = np.array([VEC_FILE_CLASSID, x.size], dtype=it).tobytes()
    # the bits as integers, so NaN payloads survive the byte swap untouched
    return head + np.ascontiguousarray(x, dtype=np.float64).view("<u8").astype(">u8").tobytes()
