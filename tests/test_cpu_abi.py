"""CPU: libfrsdg loads, exports every entry point declared in include/frsdg.h, its
ctypes mirror matches the C layout, and configuration errors are reported
without a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "frsdg.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(frsdg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "frsdg_create" in names and "frsdg_jvp" in names
    assert set(names) == set(A.SIGNATURES), "ctypes SIGNATURES out of sync with include/frsdg.h"


def test_library_exports_every_declared_symbol():
    lib = A.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (frsdg_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported
    assert lib.frsdg_abi_version() == 2


def test_struct_layout_matches_c(tmp_path):
    fields = [f[0] for f in A.frsdg_config._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
           'printf("%zu %zu\\n", sizeof(frsdg_config), sizeof(frsdg_bc));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof(frsdg_config, {f}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == C.sizeof(A.frsdg_config)
    assert vals[1] == C.sizeof(A.frsdg_bc)
    for f, off in zip(fields, vals[2:]):
        assert getattr(A.frsdg_config, f).offset == off, f


def _create(cfg):
    h = C.c_void_p()
    rc = A.lib().frsdg_create(C.byref(cfg), C.byref(h))
    if rc == A.OK:
        A.lib().frsdg_destroy(h)
    return rc


@pytest.mark.parametrize("mutate, code", [
    (lambda c: setattr(c, "poly_deg", 0), A.ERR_ARG),
    (lambda c: setattr(c, "poly_deg", 10), A.ERR_ARG),
    (lambda c: setattr(c, "dim", 3), A.ERR_ARG),
    (lambda c: c.n_elems.__setitem__(0, 1), A.ERR_ARG),
    (lambda c: setattr(c, "gamma", 1.0), A.ERR_ARG),
    (lambda c: setattr(c.bc[A.LEFT], "kind", A.BC_PERIODIC), A.ERR_ARG),  # only one side periodic
    (lambda c: (setattr(c, "apply_filter", 1), setattr(c, "filt_cut_off", 3)), A.ERR_ARG),  # 0/0 strength
    (lambda c: setattr(c, "csd_eps", 0.0), A.ERR_ARG),
    (lambda c: (setattr(c, "pp_limit", 1), setattr(c, "pp_eps", 0.0)), A.ERR_ARG),
    (lambda c: setattr(c, "coord_sys", A.COORD_RADIAL), A.ERR_UNSUPPORTED),
])
def test_invalid_configurations_rejected(mutate, code):
    cfg = make_config(dim=2, p=3, n_elems=(4, 4))
    mutate(cfg)
    assert _create(cfg) == code
    assert A.lib().frsdg_last_error()


def test_create_reports_missing_device():
    import torch

    cfg = make_config(dim=2, p=3, n_elems=(4, 4))
    rc = _create(cfg)
    assert rc == (A.OK if torch.cuda.is_available() else A.ERR_NODEVICE)


def test_null_arguments():
    lib = A.lib()
    assert lib.frsdg_create(None, None) == A.ERR_ARG
    assert lib.frsdg_residual(None, 0.0, None, None, None) == A.ERR_ARG
    assert lib.frsdg_jvp(None, None, None, None) == A.ERR_ARG
    assert lib.frsdg_status(None, None) == A.ERR_ARG
