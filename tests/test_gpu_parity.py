"""GPU parity: libfrsdg through its C ABI against the CPU oracle on seeded inputs.

Bar: max|gpu - oracle| / max|oracle| <= 1e-12 for the FP64 residual forms
(R, -R, U_t + R), the post-step stabilisation and the change of variables, and
<= 1e-11 for the complex-step JVP.
"""
import zlib

import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from oracle.oracle import Oracle
from tests.cases import CASES_1D, CASES_2D, PER, _cfg2d, cfg1d
from tests.helpers import TOL_FP64, TOL_JVP, cons_to_prim, random_state, rel_err

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.fixture(scope="module", params=sorted(CASES_2D))
def case2d(request):
    cfg = _cfg2d(**CASES_2D[request.param])
    return request.param, cfg


def test_residual_2d(case2d, cuda):
    name, cfg = case2d
    U = random_state(cfg, seed=zlib.crc32(name.encode()) % 1000)
    t = 0.7
    ref = Oracle(cfg, threads=4).residual(t, U)
    with FRSolver(cfg) as s:
        Ud = _dev(U, cuda)
        R = torch.empty_like(Ud)
        s.residual_kernel(t, Ud, R)
        got = R.cpu().numpy()
        assert s.status() == 0
    err = rel_err(got, ref)
    assert err <= TOL_FP64, f"{name}: rel err {err:.3e}"


def test_rhs_and_ifunction_2d(case2d, cuda):
    name, cfg = case2d
    U = random_state(cfg, seed=7 + zlib.crc32(name.encode()) % 97, smooth=True)
    Udot = np.random.default_rng(3).normal(size=U.size)
    o = Oracle(cfg, threads=4)
    with FRSolver(cfg) as s:
        Ud, Ut = _dev(U, cuda), _dev(Udot, cuda)
        F = torch.empty_like(Ud)
        s.rhs_func(0.3, Ud, F)
        assert rel_err(F.cpu().numpy(), o.rhs(0.3, U)) <= TOL_FP64
        s.fun_implicit(0.3, Ud, Ut, F)
        assert rel_err(F.cpu().numpy(), o.ifunction(0.3, U, Udot)) <= TOL_FP64


def test_jvp_2d(case2d, cuda):
    name, cfg = case2d
    U = random_state(cfg, seed=11)
    V = np.random.default_rng(5).normal(size=U.size)
    for h in (1e-7, 1e-30):
        cfg.csd_eps = h
        ref = Oracle(cfg, threads=4).jvp(0.2, 2.5, U, V)
        with FRSolver(cfg) as s:
            Ud, Vd = _dev(U, cuda), _dev(V, cuda)
            JV = torch.empty_like(Ud)
            s.pre_jv_eval(0.2, Ud, 2.5)
            s.matmult(Vd, JV)
            err = rel_err(JV.cpu().numpy(), ref)
        assert err <= TOL_JVP, f"{name} h={h}: rel err {err:.3e}"


@pytest.mark.parametrize("name", ["cart_ideal_hllc_p2", "sinewarp_hllc_p4_periodic", "cart_vdw_hllc_p4_walls"])
def test_change_of_variables_2d(name, cuda):
    cfg = _cfg2d(**CASES_2D[name])
    cfg.cond_sys = 1
    Uc = random_state(cfg, seed=21, smooth=True)
    P = cons_to_prim(cfg, Uc)
    Udot = np.random.default_rng(9).normal(size=P.size)
    V = np.random.default_rng(10).normal(size=P.size)
    o = Oracle(cfg, threads=4)
    with FRSolver(cfg) as s:
        Pd, Ut, Vd = _dev(P, cuda), _dev(Udot, cuda), _dev(V, cuda)
        out = torch.empty_like(Pd)
        s.primitive_to_conservative(Pd, out)
        assert rel_err(out.cpu().numpy(), o.prim_to_cons(P)) <= TOL_FP64
        s.fun_implicit(0.1, Pd, Ut, out)
        assert rel_err(out.cpu().numpy(), o.ifunction(0.1, P, Udot)) <= TOL_FP64
        for h in (1e-7, 1e-30):
            cfg.csd_eps = h
            with FRSolver(cfg) as s2:
                s2.pre_jv_eval(0.1, Pd, 1.5)
                s2.matmult(Vd, out)
                assert rel_err(out.cpu().numpy(), Oracle(cfg).jvp(0.1, 1.5, P, V)) <= TOL_JVP


@pytest.mark.parametrize("stab", ["filter", "weno", "both"])
@pytest.mark.parametrize("name", ["cart_ideal_rusanov_p3", "cart_vdw_rusanov_p5_perx", "sinewarp_hllc_p4_periodic",
                                  "cart_ideal_hllc_p7", "cart_vdw_hllc_p8_periodic"])
def test_post_step_2d(name, stab, cuda):
    kw = dict(CASES_2D[name])
    kw.update(apply_filter=stab in ("filter", "both"), apply_weno=stab in ("weno", "both"), threshold=0.3)
    cfg = _cfg2d(**kw)
    U = random_state(cfg, seed=31)
    ref = Oracle(cfg).post_step(U)
    with FRSolver(cfg) as s:
        Ud = _dev(U, cuda)
        s.apply_stabilization(Ud)
        got = Ud.cpu().numpy()
    err = rel_err(got, ref)
    assert err <= TOL_FP64, f"{name}/{stab}: rel err {err:.3e}"


# ---------------------------------------------------------------- 1D
@pytest.fixture(scope="module", params=sorted(CASES_1D))
def case1d(request):
    return request.param, cfg1d(request.param)


def test_residual_1d(case1d, cuda):
    name, cfg = case1d
    U = random_state(cfg, seed=41)
    Udot = np.random.default_rng(2).normal(size=U.size)
    V = np.random.default_rng(4).normal(size=U.size)
    o = Oracle(cfg)
    with FRSolver(cfg) as s:
        Ud, Ut, Vd = _dev(U, cuda), _dev(Udot, cuda), _dev(V, cuda)
        out = torch.empty_like(Ud)
        s.residual_kernel(0.0, Ud, out)
        assert rel_err(out.cpu().numpy(), o.residual(0.0, U)) <= TOL_FP64, name
        s.rhs_func(0.0, Ud, out)
        assert rel_err(out.cpu().numpy(), o.rhs(0.0, U)) <= TOL_FP64, name
        s.fun_implicit(0.0, Ud, Ut, out)
        assert rel_err(out.cpu().numpy(), o.ifunction(0.0, U, Udot)) <= TOL_FP64, name
        s.pre_jv_eval(0.0, Ud, 3.0)
        s.matmult(Vd, out)
        assert rel_err(out.cpu().numpy(), o.jvp(0.0, 3.0, U, V)) <= TOL_JVP, name


@pytest.mark.parametrize("stab", ["filter", "weno"])
def test_post_step_1d(case1d, stab, cuda):
    name, cfg = case1d
    cfg.apply_filter = int(stab == "filter")
    cfg.apply_weno = int(stab == "weno")
    cfg.shock_threshold = 0.3
    if cfg.apply_filter and cfg.filt_cut_off == cfg.poly_deg:
        cfg.filt_cut_off = cfg.poly_deg - 1
    U = random_state(cfg, seed=43)
    ref = Oracle(cfg).post_step(U)
    with FRSolver(cfg) as s:
        Ud = _dev(U, cuda)
        s.apply_stabilization(Ud)
        assert rel_err(Ud.cpu().numpy(), ref) <= TOL_FP64, name


def test_free_stream_preserved_large(cuda):
    """Constant state on a curved periodic mesh: R = 0 up to rounding (the
    DoNothing problem of factory.hpp:33-56 on the sine-warped mesh)."""
    cfg = _cfg2d(p=4, n_elems=(64, 64), box=(10.0, 10.0), geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                 bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER})
    with FRSolver(cfg) as s:
        U = torch.tensor([1.0, 0.5, -0.3, 2.5], dtype=torch.float64, device=cuda).repeat(s.n_dofs // 4)
        R = torch.empty_like(U)
        s.residual_kernel(0.0, U, R)
        assert R.abs().max().item() < 1e-11


@pytest.mark.parametrize("stab", ["filter", "weno"])
def test_post_step_to_equals_in_place(stab, cuda):
    """frsdg_post_step_to (src -> dst, no device copy) gives the in-place post-step's
    result bit for bit and leaves src unchanged; aliasing src and dst is refused."""
    kw = dict(CASES_2D["cart_vdw_rusanov_p5_perx"])
    kw.update(apply_filter=stab == "filter", apply_weno=stab == "weno", threshold=0.3)
    cfg = _cfg2d(**kw)
    U = _dev(random_state(cfg, seed=37), cuda)
    with FRSolver(cfg) as s:
        ref = U.clone()
        s.apply_stabilization(ref)
        src = U.clone()
        dst = torch.full_like(U, float("nan"))
        s.apply_stabilization_to(src, dst)
        torch.cuda.synchronize()
        assert torch.equal(dst, ref)
        assert torch.equal(src, U)
        assert A.lib().frsdg_post_step_to(s._h, src.data_ptr(), src.data_ptr(), None) == A.ERR_ARG


@pytest.mark.parametrize("scale", [1e-150, 1e150])
@pytest.mark.parametrize("name", ["cart_ideal_hllc_p7", "cart_ideal_rusanov_p3", "sinewarp_hllc_p4_periodic"])
def test_residual_outside_float_range(name, scale, cuda):
    """Every conservative value scaled by 1e-150 or 1e150: densities, pressures and the
    HLLC denominators leave the range where the FP64 reciprocal and square root take
    their single-precision seeds, so every node and face point is redone with the
    checked IEEE operations; the residual (R scales with the state for an ideal gas)
    still equals the oracle's."""
    cfg = _cfg2d(**CASES_2D[name])
    U = random_state(cfg, seed=77) * scale
    ref = Oracle(cfg, threads=4).residual(0.2, U)
    assert np.all(np.isfinite(ref))
    with FRSolver(cfg) as s:
        Ud = _dev(U, cuda)
        R = torch.empty_like(Ud)
        s.residual_kernel(0.2, Ud, R)
        got = R.cpu().numpy()
        assert s.status() == 0
    err = rel_err(got, ref)
    assert err <= TOL_FP64, f"{name} x {scale:g}: rel err {err:.3e}"
