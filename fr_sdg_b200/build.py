"""Build libfrsdg.so (the CUDA library behind include/frsdg.h) for sm_100a.

Compiles every translation unit under fr_sdg_b200/csrc with nvcc in parallel
into fr_sdg_b200/_build/ and links fr_sdg_b200/libfrsdg.so.  Objects are
rebuilt only when a source or header is newer than the object.

    python -m fr_sdg_b200.build [-j JOBS] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libfrsdg.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]
N_VALUES = range(2, 11)  # GLL points per direction, p = 1..9


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _units() -> list[tuple[Path, Path, list[str]]]:
    units = []
    for n in N_VALUES:
        units.append((CSRC / "instances.cu", BUILD / f"instances_n{n}.o", [f"-DFRSDG_N={n}"]))
    for name in ("capi.cu", "stab.cu", "setup_ops.cpp", "noalloc.cu", "jacobi.cu", "petsc_io.cu", "pplimit.cu", "batch.cu", "tc.cu", "krylov.cu"):
        units.append((CSRC / name, BUILD / (Path(name).stem + ".o"), []))
    return units


def _headers_mtime() -> float:
    files = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [INCLUDE / "frsdg.h"]
    return max(f.stat().st_mtime for f in files)


def _compile(nvcc: str, src: Path, obj: Path, extra: list[str], force: bool) -> str:
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _headers_mtime()):
        return f"up to date {obj.name}"
    cmd = [nvcc, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [nvcc, *NVCC_FLAGS, "-x", "cu", *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return f"built {obj.name}"


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    units = _units()
    jobs = jobs or max(1, min(len(units), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, nvcc, s, o, e, force) for s, o, e in units]
        for f in cf.as_completed(futs):
            msg = f.result()
            if verbose:
                print(msg, flush=True)
    objs = [str(o) for _, o, _ in units]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
        if verbose:
            print(f"linked {LIB}", flush=True)
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    build(args.jobs, args.force, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
