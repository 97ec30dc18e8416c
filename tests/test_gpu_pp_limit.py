"""GPU: frsdg_pp_limit (the positivity-preserving limiter; no counterpart in the
reference) and the post-step that ends with it, through the C ABI against the oracle
on states whose nodes are inadmissible: max|gpu - oracle| / max|oracle| <= 1e-12."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from oracle.oracle import Oracle
from tests.cases import CASES_2D, _cfg2d, cfg1d
from tests.helpers import TOL_FP64, poisoned_state, random_state, rel_err

pytestmark = pytest.mark.gpu

NAMES_2D = ["cart_ideal_rusanov_p3", "cart_vdw_rusanov_p5_perx", "sinewarp_hllc_p4_periodic",
            "bump_hllc_p3_inflow_outlet", "cart_ideal_hllc_p7", "cart_ideal_hllc_p1_periodic"]


def _dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("name", NAMES_2D)
def test_pp_limit_2d(name, cuda):
    cfg = _cfg2d(**CASES_2D[name], pp_limit=True)
    U = poisoned_state(cfg, seed=11)
    ref = Oracle(cfg).pp_limit(U)
    with FRSolver(cfg) as s:
        X = _dev(U, cuda)
        s.pp_limit(X)
        assert rel_err(X.cpu().numpy(), ref) <= TOL_FP64
        # admissible input: untouched, bit for bit
        V = _dev(random_state(cfg, seed=12), cuda)
        W = V.clone()
        s.pp_limit(W)
        assert torch.equal(V, W)


def test_pp_limit_refreshes_the_fp32_copy(cuda):
    cfg = _cfg2d(**CASES_2D["cart_vdw_rusanov_p5_perx"], pp_limit=True)
    U = poisoned_state(cfg, seed=13)
    with FRSolver(cfg) as s:
        X = _dev(U, cuda)
        X32 = X.float()
        s.pp_limit(X, X32)
        assert torch.equal(X32, X.float())


@pytest.mark.parametrize("name", ["sod_rusanov_p3", "vdw_hllc_p5_walls", "p9_rusanov"])
def test_pp_limit_1d(name, cuda):
    cfg = cfg1d(name, pp_limit=True)
    U = poisoned_state(cfg, seed=14)
    ref = Oracle(cfg).pp_limit(U)
    with FRSolver(cfg) as s:
        X = _dev(U, cuda)
        s.pp_limit(X)
        assert rel_err(X.cpu().numpy(), ref) <= TOL_FP64


@pytest.mark.parametrize("stab", ["none", "filter", "weno", "both"])
@pytest.mark.parametrize("name", ["cart_ideal_rusanov_p3", "sinewarp_hllc_p4_periodic", "cart_vdw_hllc_p8_periodic"])
def test_post_step_with_limiter(name, stab, cuda):
    kw = dict(CASES_2D[name])
    kw.update(apply_filter=stab in ("filter", "both"), apply_weno=stab in ("weno", "both"), threshold=0.3,
              pp_limit=True)
    cfg = _cfg2d(**kw)
    U = poisoned_state(cfg, seed=15)
    ref = Oracle(cfg).post_step(U)
    with FRSolver(cfg) as s:
        X = _dev(U, cuda)
        s.apply_stabilization(X)
        assert rel_err(X.cpu().numpy(), ref) <= TOL_FP64
        src, dst = _dev(U, cuda), torch.empty_like(X)
        s.apply_stabilization_to(src, dst)
        assert rel_err(dst.cpu().numpy(), ref) <= TOL_FP64


def test_static_post_step_rejects_the_limiter(cuda):
    cfg = _cfg2d(**CASES_2D["cart_ideal_rusanov_p3"], apply_filter=True, pp_limit=True)
    X = _dev(random_state(cfg, seed=16), cuda)
    assert A.lib().frsdg_post_step_static(cfg, X.data_ptr(), None) == A.ERR_UNSUPPORTED


def test_blast_runs_finite_with_limiter(cuda):
    """The blast workload (filter with the shock sensor, positivity limiter, CFL 0.1 with
    the (2p+1) rule) on a 64^2 p5 mesh: 100 SSP-RK3 steps keep every node admissible."""
    from fr_sdg_b200.integrate import Integrator
    from fr_sdg_b200.workloads import blast_large

    wl = blast_large(64, 5)
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        dt = wl.time_step(U)
        Integrator(s, "ssprk3").run(U, dt, n_steps=100)
        q = U.view(-1, 4)
        assert bool(torch.isfinite(U).all()) and float(q[:, 0].min()) > 0.0
        assert s.status() == 0
