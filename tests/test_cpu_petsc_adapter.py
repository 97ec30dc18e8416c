"""CPU: the PETSc adapter (fr_sdg_b200/petsc/frsdg_petsc.cpp) compiles against the PETSc
API it binds and against the library's C ABI.

PETSc is not installed here, so the adapter is compiled against tests/petsc_decl/, a
declaration-only copy of the PETSc 3.21 signatures it uses (TS callbacks, MatShell,
DMDA corners, CUDA Vec arrays), with all warnings as errors.  The object must define
every function include/frsdg_petsc.h declares, with C linkage, and every libfrsdg
entry point it calls must be exported by the built library."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CUDA_INC = Path("/usr/local/cuda/include")


def _tools():
    if shutil.which("g++") is None or shutil.which("nm") is None or not (CUDA_INC / "cuda_runtime.h").exists():
        pytest.skip("g++, nm or the CUDA runtime headers are missing")


@pytest.fixture(scope="module")
def adapter_object(tmp_path_factory):
    _tools()
    out = tmp_path_factory.mktemp("petsc") / "frsdg_petsc.o"
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-O2", "-fPIC", "-c",
           "-I", str(ROOT / "tests" / "petsc_decl"), "-I", str(ROOT / "include"), "-I", str(CUDA_INC),
           str(ROOT / "fr_sdg_b200" / "petsc" / "frsdg_petsc.cpp"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return out


def _symbols(obj: Path, undefined: bool) -> set[str]:
    flag = "--undefined-only" if undefined else "--defined-only"
    res = subprocess.run(["nm", "-g", flag, str(obj)], capture_output=True, text=True, check=True)
    return {ln.split()[-1] for ln in res.stdout.splitlines() if ln.strip()}


def test_adapter_defines_every_declared_function(adapter_object):
    header = (ROOT / "include" / "frsdg_petsc.h").read_text()
    declared = set(re.findall(r"^\w[\w\s\*]*?\b(FrsdgPetsc\w+)\(", header, flags=re.M))
    assert len(declared) == 13, sorted(declared)
    assert declared <= _symbols(adapter_object, undefined=False)  # unmangled: C linkage


def test_adapter_calls_only_exported_library_entry_points(adapter_object):
    lib = ROOT / "fr_sdg_b200" / "libfrsdg.so"
    if not lib.exists():
        pytest.skip("libfrsdg.so is not built")
    used = {s for s in _symbols(adapter_object, undefined=True) if s.startswith("frsdg_")}
    assert {"frsdg_rhs", "frsdg_ifunction", "frsdg_jvp_prepare", "frsdg_jvp", "frsdg_post_step",
            "frsdg_post_step_to", "frsdg_prim_to_cons", "frsdg_set_row_window"} <= used
    res = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True)
    exported = {ln.split()[-1] for ln in res.stdout.splitlines() if ln.strip()}
    assert used <= exported, sorted(used - exported)
