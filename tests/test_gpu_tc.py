"""GPU: the split-precision tensor-core line contraction (tcgen05, TF32 high and low
parts, FP32 accumulation) against FP64 products: every derivative within a few FP32
units of the sum of |D_km v_m|, for the GLL differentiation matrices p = 1..7 and for
random matrices, on line counts that leave partial MMA tiles."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import _abi as A
from fr_sdg_b200.refelem import reference_element

pytestmark = pytest.mark.gpu

# FP32 accuracy: hi + lo keeps 22 significant bits of each operand; the three products
# are exact and their FP32 sums add a few units of 2^-24 of the magnitude.
REL_TOL = 2.0 ** -20


def _contract(v: np.ndarray, D: np.ndarray, cuda) -> np.ndarray:
    n = D.shape[0]
    vd = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).to(cuda)
    Dd = torch.from_numpy(np.array(D, dtype=np.float64)).to(cuda)
    out = torch.full_like(vd, float("nan"))
    A.check(A.lib().frsdg_tc_lines(n, vd.data_ptr(), Dd.data_ptr(), out.data_ptr(), v.shape[0], None),
            "frsdg_tc_lines")
    return out.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("lines", [1, 191, 192, 193, 1000])
def test_gll_derivatives(p, lines, cuda):
    _, _, D, _, _ = reference_element(p)
    rng = np.random.default_rng(100 * p + lines)
    v = rng.uniform(-3.0, 3.0, size=(lines, p + 1)).astype(np.float32)
    got = _contract(v, D, cuda)
    vv = v.astype(np.float64)
    ref = vv @ D.T
    scale = np.abs(vv) @ np.abs(D).T
    assert np.all(np.abs(got - ref) <= REL_TOL * scale + 1e-30)


@pytest.mark.parametrize("n", [2, 5, 6, 8])
def test_random_matrices_and_magnitudes(n, cuda):
    rng = np.random.default_rng(n)
    D = rng.normal(size=(n, n)) * 10.0 ** rng.integers(-3, 4, size=(n, n))
    v = (rng.normal(size=(777, n)) * 10.0 ** rng.integers(-5, 6, size=(777, 1))).astype(np.float32)
    got = _contract(v, D, cuda)
    vv = v.astype(np.float64)
    ref = vv @ D.T
    scale = np.abs(vv) @ np.abs(D).T
    assert np.all(np.abs(got - ref) <= REL_TOL * scale + 1e-30)


def test_rejects_bad_arguments(cuda):
    lib = A.lib()
    x = torch.zeros(8, device=cuda)
    assert lib.frsdg_tc_lines(9, x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, None) == A.ERR_ARG
    assert lib.frsdg_tc_lines(1, x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, None) == A.ERR_ARG
    assert lib.frsdg_tc_lines(4, None, x.data_ptr(), x.data_ptr(), 1, None) == A.ERR_ARG
    assert lib.frsdg_tc_lines(4, None, None, None, 0, None) == A.OK
