"""GPU: libfrsdg through its C ABI against outputs of fr_sdg's OWN hot-path code.

tests/golden/ref_<case>.npz were written by the reference's include/*.hpp compiled
into oracle/_ref/libfrsdg_ref.so (tests/golden/gen_ref_golden.py).  The CUDA path
must reproduce them within the parity bars: 1e-12 relative for the FP64 forms, the
JVP tolerance for the complex step.
"""
from pathlib import Path

import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from tests.cases import REF_FIXTURES_1D, REF_FIXTURES_2D, ref_fixture_cfg
from tests.helpers import TOL_FP64, TOL_JVP, rel_err

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
FIXTURES = list(REF_FIXTURES_2D) + ["1d_" + n for n in REF_FIXTURES_1D]


def _dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("name", FIXTURES)
def test_cuda_reproduces_reference_fixture(name, cuda):
    d = np.load(GOLD / f"ref_{name}.npz")
    cfg = ref_fixture_cfg(name)
    U, V, Udot = (_dev(d[k], cuda) for k in ("U", "V", "Udot"))
    out = torch.empty_like(U)
    with FRSolver(cfg) as s:
        s.residual_kernel(0.7, U, out)
        assert rel_err(out.cpu().numpy(), d["R"]) <= TOL_FP64
        s.fun_implicit(0.3, U, Udot, out)
        assert rel_err(out.cpu().numpy(), d["IF"]) <= TOL_FP64
        assert s.status() == 0
    for h, key in ((1e-7, "JV7"), (1e-30, "JV30")):
        cfg.csd_eps = h
        with FRSolver(cfg) as s:
            s.pre_jv_eval(0.2, U, 2.5)
            s.matmult(V, out)
            assert rel_err(out.cpu().numpy(), d[key]) <= TOL_JVP, key
    cfg.csd_eps = 1e-7
    if cfg.filt_cut_off >= cfg.poly_deg:
        cfg.filt_cut_off = max(cfg.poly_deg - 1, 0)
    for key, (f, w) in (("POSTF", (1, 0)), ("POSTW", (0, 1)), ("POSTB", (1, 1))):
        cfg.apply_filter, cfg.apply_weno, cfg.shock_threshold = f, w, 0.3
        with FRSolver(cfg) as s:
            X = U.clone()
            s.apply_stabilization(X)
            assert rel_err(X.cpu().numpy(), d[key]) <= TOL_FP64, key
    if "P" in d:
        c2 = ref_fixture_cfg(name, cond_sys=True)
        P = _dev(d["P"], cuda)
        with FRSolver(c2) as s:
            s.primitive_to_conservative(P, out)
            assert rel_err(out.cpu().numpy(), d["CONS"]) <= TOL_FP64
            s.fun_implicit(0.1, P, Udot, out)
            assert rel_err(out.cpu().numpy(), d["IFC"]) <= TOL_FP64
            s.pre_jv_eval(0.1, P, 1.5)
            s.matmult(V, out)
            assert rel_err(out.cpu().numpy(), d["JVC"]) <= TOL_JVP
