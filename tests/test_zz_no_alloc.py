"""GPU: frsdg_post_step_static, the post-step entry point that allocates nothing.

A caller that cannot allocate device memory at the time it limits a solution
(while a stream is being captured into a CUDA graph, or under a memory manager
that owns every allocation) calls this entry point with the configuration
instead of a handle; the copy the WENO limiter reads from is a fixed array
inside the library.  These tests call it through the C ABI twice in a row and
compare each result with frsdg_post_step on the same input.  This file is named
so that pytest collects it last.
"""
import ctypes as C

import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config
from tests.helpers import TOL_FP64, random_state, rel_err

pytestmark = pytest.mark.gpu


def _static(cfg, U: torch.Tensor) -> None:
    rc = A.lib().frsdg_post_step_static(C.byref(cfg), U.data_ptr(), torch.cuda.current_stream().cuda_stream)
    A.check(rc, "frsdg_post_step_static")


@pytest.mark.parametrize("dim", [2, 1])
@pytest.mark.parametrize("stab", ["weno", "filter", "both"])
def test_static_post_step_matches_handle(dim, stab, cuda):
    if dim == 2:
        cfg = make_config(dim=2, p=4, n_elems=(9, 7), box=(1.0, 1.0), riemann="hllc",
                          bcs={A.LEFT: A.BC_PERIODIC, A.RIGHT: A.BC_PERIODIC, A.TOP: A.BC_WALL,
                               A.BOTTOM: A.BC_OUTFLOW})
    else:
        cfg = make_config(dim=1, p=3, n_elems=(40, 1), riemann="rusanov",
                          bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW})
    cfg.apply_filter = int(stab in ("filter", "both"))
    cfg.apply_weno = int(stab in ("weno", "both"))
    cfg.shock_threshold = 0.3
    # two calls in a row, on different inputs, each against the handle's entry point
    for seed in (5, 6):
        U0 = torch.from_numpy(random_state(cfg, seed=seed)).to(cuda)
        ref = U0.clone()
        with FRSolver(cfg) as s:
            s.apply_stabilization(ref)
        got = U0.clone()
        _static(cfg, got)
        torch.cuda.synchronize()
        err = rel_err(got.cpu().numpy(), ref.cpu().numpy())
        assert err <= TOL_FP64, f"{dim}D {stab} seed {seed}: rel err {err:.3e}"


def test_static_post_step_rejects_oversize(cuda):
    n_side = 300  # 300*300*4*16 doubles > FRSDG_POST_STEP_STATIC_MAX_DOFS
    cfg = make_config(dim=2, p=3, n_elems=(n_side, n_side), apply_weno=True)
    assert n_side * n_side * 64 > A.POST_STEP_STATIC_MAX_DOFS
    U = torch.empty(1, dtype=torch.float64, device=cuda)
    rc = A.lib().frsdg_post_step_static(C.byref(cfg), U.data_ptr(), None)
    assert rc == A.ERR_ARG
    assert b"FRSDG_POST_STEP_STATIC_MAX_DOFS" in A.lib().frsdg_last_error()


@pytest.mark.parametrize("dim", [2, 1])
def test_static_post_step_replays_in_a_cuda_graph(dim, cuda):
    """The use the entry point exists for: after one warm-up call outside capture, the
    WENO post-step is captured into a CUDA graph (no allocation is allowed there) and
    every replay limits the graph's input buffer exactly as frsdg_post_step does."""
    if dim == 2:
        cfg = make_config(dim=2, p=3, n_elems=(8, 6), box=(1.0, 1.0), riemann="hllc",
                          bcs={A.LEFT: A.BC_PERIODIC, A.RIGHT: A.BC_PERIODIC, A.TOP: A.BC_WALL,
                               A.BOTTOM: A.BC_OUTFLOW})
    else:
        cfg = make_config(dim=1, p=4, n_elems=(32, 1), riemann="rusanov",
                          bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW})
    cfg.apply_weno = 1
    cfg.shock_threshold = 0.3
    buf = torch.from_numpy(random_state(cfg, seed=40)).to(cuda)
    _static(cfg, buf.clone())  # warm-up: the scratch address is looked up outside capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        _static(cfg, buf)
    for seed in (41, 42):
        U0 = torch.from_numpy(random_state(cfg, seed=seed)).to(cuda)
        buf.copy_(U0)
        g.replay()
        ref = U0.clone()
        with FRSolver(cfg) as s:
            s.apply_stabilization(ref)
        torch.cuda.synchronize()
        err = rel_err(buf.cpu().numpy(), ref.cpu().numpy())
        assert err <= TOL_FP64, f"{dim}D seed {seed}: rel err {err:.3e}"
    del g
