"""GPU: the host-vector entry point (frsdg_rhs_host) returns the device rhs bit for bit
-- pipelined over row chunks on 2D meshes (periodic and not), in one piece in 1D."""
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config, sod1d
from tests.helpers import random_state

pytestmark = pytest.mark.gpu

PER = (A.BC_PERIODIC, None, None)


@pytest.mark.parametrize("name,kw", [
    ("wall_outflow_p3_40x37", dict(p=3, n_elems=(40, 37), riemann="hllc",
                                   bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_WALL,
                                        A.BOTTOM: A.BC_WALL})),
    ("periodic_vdw_p5_16x64", dict(p=5, n_elems=(16, 64), riemann="hllc", gas="vdw", vdw=(0.05, 0.02),
                                   bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER})),
    ("small_p2_6x5", dict(p=2, n_elems=(6, 5), riemann="rusanov",
                          bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_OUTFLOW,
                               A.BOTTOM: A.BC_OUTFLOW})),
])
def test_rhs_host_matches_device(name, kw, cuda):
    cfg = make_config(dim=2, **kw)
    U = random_state(cfg, 17, amp=0.3)
    with FRSolver(cfg) as s:
        Ud = torch.from_numpy(U).to(cuda)
        Fd = torch.empty_like(Ud)
        s.rhs_func(0.4, Ud, Fd)
        Uh = torch.from_numpy(U).pin_memory()
        Fh = torch.full_like(Uh, float("nan")).pin_memory()
        for _ in range(2):  # the second call reuses the pipeline's streams and events
            s.rhs_func_host(0.4, Uh, Fh)
            assert torch.equal(Fh, Fd.cpu()), name


def test_rhs_host_1d(cuda):
    wl = sod1d()
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        F = torch.empty_like(U)
        s.rhs_func(0.0, U, F)
        Fh = torch.empty(U.numel(), dtype=torch.float64).pin_memory()
        s.rhs_func_host(0.0, U.cpu().pin_memory(), Fh)
        assert torch.equal(Fh, F.cpu())
