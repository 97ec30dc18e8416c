"""GPU: frsdg_rk_stage_fused -- the Runge-Kutta stage with the positivity limiter and the
element-local post-step (spectral filter, limiter) in its epilogue -- against the
unfused sequence (frsdg_rk_stage, then frsdg_post_step_to / frsdg_pp_limit) on the same
inputs.  The fused kernel computes the same values in another kernel, where the
compiler may contract other products into FMAs, so the two agree to rounding: 1e-13 of
max|out| in FP64; the WENO-only and 1D configurations take the unfused path inside the
call and agree bit for bit."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config
from tests.helpers import poisoned_state, random_state, rel_err

pytestmark = pytest.mark.gpu

PER = (A.BC_PERIODIC, None, None)
OUT = A.BC_OUTFLOW
CASES = {
    "cart_vdw_hllc_p5_periodic": dict(dim=2, p=5, n_elems=(9, 7), riemann="hllc", gas="vdw", vdw=(0.05, 0.02),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "cart_ideal_rusanov_p3_walls": dict(dim=2, p=3, n_elems=(11, 6), box=(1.3, 0.9), riemann="rusanov",
                                        bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: A.BC_WALL, A.BOTTOM: A.BC_WALL}),
    "sinewarp_hllc_p4_periodic": dict(dim=2, p=4, n_elems=(6, 6), box=(10.0, 10.0), riemann="hllc",
                                      geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "cart_ideal_hllc_p2_1d": dict(dim=1, p=2, n_elems=(40, 1), riemann="hllc", bcs={A.LEFT: OUT, A.RIGHT: OUT}),
}
STABS = {"filter_pp": dict(apply_filter=1, pp_limit=1), "pp": dict(pp_limit=1), "filter": dict(apply_filter=1),
         "weno_pp": dict(apply_weno=1, pp_limit=1)}


def _cfg(name, stab):
    cfg = make_config(**CASES[name])
    for k, v in STABS[stab].items():
        setattr(cfg, k, v)
    cfg.shock_threshold = 0.3
    cfg.filt_cut_off = min(cfg.filt_cut_off, cfg.poly_deg - 1)  # cut-off = p gives 0/0 (rejected)
    return cfg


def _inputs(cfg, cuda):
    d = lambda v: torch.from_numpy(np.ascontiguousarray(v)).to(cuda)
    Us = d(random_state(cfg, 31, amp=0.2))
    A0 = d(poisoned_state(cfg, 32))  # inadmissible nodes: the limiter acts
    B0 = d(random_state(cfg, 33, amp=0.2))
    return Us, A0, B0


@pytest.mark.parametrize("stab", sorted(STABS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_post_step_matches_separate_passes(name, stab, cuda):
    cfg = _cfg(name, stab)
    # the unfused path inside the call: the post-step in 1D and with WENO alone; the
    # limiter alone in 1D
    exact = cfg.dim == 1 or (cfg.apply_weno and not cfg.apply_filter)
    exact_limit = cfg.dim == 1
    with FRSolver(cfg) as s:
        Us, A0, B0 = _inputs(cfg, cuda)
        kw = dict(gamma=1e-3, a=A0, alpha=1.0, b=B0, beta=1e-3)
        got = torch.empty_like(Us)
        s.rk_stage_fused(0.1, Us, got, A.STAGE_POST_STEP, **kw)
        mid, ref = torch.empty_like(Us), torch.empty_like(Us)
        s.rk_stage(0.1, Us, mid, **kw)
        s.apply_stabilization_to(mid, ref)
        # the limiter alone on a stage output
        got2, ref2 = torch.empty_like(Us), torch.empty_like(Us)
        s.rk_stage_fused(0.1, Us, got2, A.STAGE_LIMIT, **kw)
        s.rk_stage(0.1, Us, ref2, **kw)
        s.pp_limit(ref2)
        torch.cuda.synchronize()
        assert s.status() == 0
    g, r = got.cpu().numpy(), ref.cpu().numpy()
    assert np.all(np.isfinite(g))
    if exact:
        assert np.array_equal(g, r)
    else:
        assert rel_err(g, r) <= 1e-13, f"{name} {stab}: post-step rel err {rel_err(g, r):.3e}"
    if exact_limit:
        assert np.array_equal(got2.cpu().numpy(), ref2.cpu().numpy())
    else:
        e2 = rel_err(got2.cpu().numpy(), ref2.cpu().numpy())
        assert e2 <= 1e-13, f"{name} {stab}: limiter rel err {e2:.3e}"
    if cfg.pp_limit:
        # the limiter did act: the unlimited stage output differs
        assert not np.array_equal(mid.cpu().numpy(), ref2.cpu().numpy())


def test_fused_stage_in_place_and_mixed(cuda):
    """out may be the state itself (the last stage writes U), and the mixed form's fused
    stage equals frsdg_rk_stage_mixed followed by the post-step."""
    cfg = _cfg("cart_vdw_hllc_p5_periodic", "filter_pp")
    with FRSolver(cfg) as s:
        Us, A0, B0 = _inputs(cfg, cuda)
        kw = dict(gamma=1e-3, alpha=1.0, b=B0, beta=1e-3)
        U = A0.clone()
        s.rk_stage_fused(0.1, Us, U, A.STAGE_POST_STEP, a=U, **kw)
        mid, ref = torch.empty_like(Us), torch.empty_like(Us)
        s.rk_stage(0.1, Us, mid, a=A0, **kw)
        s.apply_stabilization_to(mid, ref)
        assert rel_err(U.cpu().numpy(), ref.cpu().numpy()) <= 1e-13
        got = torch.empty_like(Us)
        s.rk_stage_fused(0.1, Us, got, A.STAGE_POST_STEP | A.STAGE_MIXED, a=A0, **kw)
        s.rk_stage_mixed(0.1, Us, mid, a=A0, **kw)
        s.apply_stabilization_to(mid, ref)
        torch.cuda.synchronize()
        assert rel_err(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-9
        assert s.status() == 0


def test_fused_stage_rejects_bad_flags(cuda):
    cfg = _cfg("cart_ideal_rusanov_p3_walls", "pp")
    with FRSolver(cfg) as s:
        Us = torch.from_numpy(random_state(cfg, 1)).to(cuda)
        out = torch.empty_like(Us)
        with pytest.raises(RuntimeError, match="unknown flags"):
            s.rk_stage_fused(0.0, Us, out, 64, gamma=1.0)
        with pytest.raises(RuntimeError, match="alias"):
            s.rk_stage_fused(0.0, Us, Us, A.STAGE_LIMIT, gamma=1.0)
