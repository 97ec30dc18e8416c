"""GPU: the mixed-precision form -- the FP32 residual against the FP64 oracle on the
same rounded state, the mixed RK stage (FP32 residual arithmetic on an FP64 state whose
node primitives are recovered in FP64, FP64 combination), and whole vortex runs
against their FP64 twins and the exact solution."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.integrate import Integrator, cfl_time_step, l2_error, node_jacobian
from fr_sdg_b200.workloads import exact_vortex, make_config, node_coords, pack2d, vortex_curved
from oracle.oracle import Oracle
from tests.helpers import TOL_FP32, gas_rhoE, random_state, rel_err

pytestmark = pytest.mark.gpu

PER = (A.BC_PERIODIC, None, None)
OUT = A.BC_OUTFLOW
CASES = {
    "cart_ideal_hllc_p3": dict(p=3, n_elems=(7, 5), box=(1.3, 0.9), riemann="hllc",
                               bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: A.BC_WALL, A.BOTTOM: OUT}),
    "cart_vdw_rusanov_p5_periodic": dict(p=5, n_elems=(6, 4), riemann="rusanov", gas="vdw", vdw=(0.05, 0.02),
                                         bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "sinewarp_hllc_p4_periodic": dict(p=4, n_elems=(6, 6), box=(10.0, 10.0), riemann="hllc",
                                      geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "bump_hllc_p3_inflow_outlet": dict(p=3, n_elems=(12, 4), box=(3.0, 0.8), riemann="hllc",
                                       geometry=A.GEOM_WALL_PROFILE, profile=A.PROFILE_GAUSS_BUMP,
                                       geom_params=(-1.5, 0.0625, 25.0, 0.0),
                                       bcs={A.LEFT: (A.BC_SUBSONIC_INFLOW, None, (1.0, 1.0, 1.0, 0.0)),
                                            A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (0.84,)),
                                            A.BOTTOM: A.BC_SLIP_WALL, A.TOP: A.BC_SLIP_WALL}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_residual_f32_matches_oracle(name, cuda):
    cfg = make_config(dim=2, **CASES[name])
    U32 = random_state(cfg, 21, amp=0.3).astype(np.float32)
    ref = Oracle(cfg, threads=4).residual(0.2, U32.astype(np.float64))
    with FRSolver(cfg) as s:
        Ud = torch.from_numpy(U32).to(cuda)
        R = torch.empty_like(Ud)
        s.residual_kernel_f32(0.2, Ud, R)
        got = R.cpu().numpy()
    err = rel_err(got, ref)
    assert err <= TOL_FP32, f"{name}: FP32 residual rel err {err:.3e}"


def test_rk_stage_mixed_combines_in_fp64(cuda):
    cfg = make_config(dim=2, **CASES["sinewarp_hllc_p4_periodic"])
    U = random_state(cfg, 3, amp=0.2)
    rng = np.random.default_rng(4)
    Av, Bv, C0 = rng.uniform(-1, 1, U.size), rng.uniform(-1, 1, U.size), rng.uniform(-1, 1, U.size)
    alpha, beta, gamma, delta = 0.75, 0.25, 0.013, 0.007
    rhs = -Oracle(cfg, threads=4).residual(0.0, U)
    with FRSolver(cfg) as s:
        d = lambda v: torch.from_numpy(np.ascontiguousarray(v)).to(cuda)
        out, acc = torch.empty(U.size, dtype=torch.float64, device=cuda), d(C0)
        s.rk_stage_mixed(0.0, d(U), out, gamma=gamma, a=d(Av), alpha=alpha, b=d(Bv), beta=beta,
                         acc=acc, delta=delta)
        o, ac = out.cpu().numpy(), acc.cpu().numpy()
    ref = alpha * Av + beta * Bv + gamma * rhs
    assert np.max(np.abs(o - ref)) <= TOL_FP32 * gamma * np.max(np.abs(rhs))
    assert np.max(np.abs(ac - (C0 + delta * rhs))) <= TOL_FP32 * delta * np.max(np.abs(rhs))


@pytest.mark.parametrize("name", ["cart_ideal_hllc_p3", "cart_vdw_rusanov_p5_periodic"])
def test_rk_stage_mixed_recovers_primitives_in_fp64(name, cuda):
    """A fast, cold flow (kinetic energy 1e6 times the internal energy): rounded to FP32,
    rho E minus the kinetic energy is rounding noise and the pressure's sign is lost; the
    mixed stage recovers every node's pressure and sound speed from the FP64 state, so
    its residual stays finite and within the FP32 tolerance of the FP64 oracle."""
    cfg = make_config(dim=2, **CASES[name])
    n = cfg.poly_deg + 1
    nodes = cfg.n_elems[0] * cfg.n_elems[1] * n * n
    r = np.random.default_rng(8).uniform(-1, 1, size=(nodes, 4))
    rho = 1.0 + 0.1 * r[:, 0]
    u, v = 10.0 + 0.3 * r[:, 1], 0.3 * r[:, 2]
    p = 1e-4 * (1.0 + 0.5 * r[:, 3])
    E = gas_rhoE(cfg, rho, u * u + v * v, p)
    U = np.stack([rho, rho * u, rho * v, E], axis=1).reshape(-1)
    rhs = -Oracle(cfg, threads=4).residual(0.0, U)
    assert np.all(np.isfinite(rhs))
    with FRSolver(cfg) as s:
        Ud = torch.from_numpy(U).to(cuda)
        out = torch.empty_like(Ud)
        s.rk_stage_mixed(0.0, Ud, out, gamma=1.0)
        got = out.cpu().numpy()
        assert s.status() == 0
    assert np.all(np.isfinite(got))
    err = rel_err(got, rhs)
    assert err <= TOL_FP32, f"{name}: mixed stage rel err {err:.3e}"


@pytest.mark.parametrize("ne", [16, 32])
def test_mixed_vortex_matches_fp64_accuracy(ne, cuda):
    """Curved isentropic vortex, p = 4, RK4 to t = 1: the mixed-precision run's L2
    density error against the exact solution is within 10 % of the FP64 run's."""
    wl = vortex_curved(n_elems=ne, p=4)
    errs = {}
    with FRSolver(wl.cfg) as s:
        x, y = node_coords(wl.cfg, cuda)
        ex = pack2d(*exact_vortex(1.0, x, y))
        J = node_jacobian(wl.cfg, cuda)
        for mixed in (False, True):
            U = wl.init(cuda)
            dt = cfl_time_step(wl.cfg, U, 0.05)
            Integrator(s, "rk4", mixed=mixed).run(U, dt, t_end=1.0)
            errs[mixed] = float(l2_error(wl.cfg, U, ex, J)[0])
        assert s.status() == 0
    assert errs[True] <= 1.1 * errs[False], errs


# ---- the FP32 residual with its derivative contractions on the tensor cores --------
# (cfg.mixed_tc = 1, p = 4 to 7).  Meshes whose sizes leave partial tiles on both axes.
TC_CASES = {
    "cart_vdw_hllc_p4_walls": dict(p=4, n_elems=(9, 5), box=(1.3, 0.9), riemann="hllc", gas="vdw",
                                   vdw=(0.05, 0.02),
                                   bcs={A.LEFT: OUT, A.RIGHT: A.BC_WALL, A.TOP: A.BC_WALL, A.BOTTOM: OUT}),
    "cart_vdw_rusanov_p5_periodic": dict(p=5, n_elems=(7, 5), riemann="rusanov", gas="vdw", vdw=(0.05, 0.02),
                                         bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "sinewarp_hllc_p4_periodic": CASES["sinewarp_hllc_p4_periodic"],
    "sinewarp_rusanov_p5_periodic": dict(p=5, n_elems=(5, 7), box=(10.0, 10.0), riemann="rusanov",
                                         geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                         bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "bump_hllc_p5_inflow_outlet": dict(CASES["bump_hllc_p3_inflow_outlet"], p=5, n_elems=(11, 3)),
    "cart_vdw_hllc_p6_walls": dict(p=6, n_elems=(5, 3), box=(1.3, 0.9), riemann="hllc", gas="vdw",
                                   vdw=(0.05, 0.02),
                                   bcs={A.LEFT: OUT, A.RIGHT: A.BC_WALL, A.TOP: A.BC_WALL, A.BOTTOM: OUT}),
    "sinewarp_hllc_p7_periodic": dict(p=7, n_elems=(3, 5), box=(10.0, 10.0), riemann="hllc",
                                      geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
}


def _tc_cfg(name, tc=1):
    cfg = make_config(dim=2, **TC_CASES[name])
    cfg.mixed_tc = tc
    return cfg


@pytest.mark.parametrize("name", sorted(TC_CASES))
def test_residual_f32_tensor_cores_match_oracle(name, cuda):
    """The tensor-core FP32 residual against the FP64 oracle (FP32 tolerance) and against
    the CUDA-core FP32 residual (the same arithmetic but for the contraction order)."""
    cfg = _tc_cfg(name)
    U32 = random_state(cfg, 31, amp=0.3).astype(np.float32)
    ref = Oracle(cfg, threads=4).residual(0.2, U32.astype(np.float64))
    got = {}
    for tc in (1, 0):
        cfg.mixed_tc = tc
        with FRSolver(cfg) as s:
            Ud = torch.from_numpy(U32).to(cuda)
            R = torch.full_like(Ud, float("nan"))
            s.residual_kernel_f32(0.2, Ud, R)
            got[tc] = R.cpu().numpy()
            assert s.status() == 0
    err = rel_err(got[1], ref)
    assert err <= TOL_FP32, f"{name}: tensor-core FP32 residual rel err {err:.3e}"
    assert rel_err(got[1], got[0]) <= TOL_FP32


@pytest.mark.parametrize("name", ["cart_vdw_hllc_p4_walls", "sinewarp_rusanov_p5_periodic"])
def test_fused_mixed_stage_with_tensor_cores(name, cuda):
    """A mixed stage with the filter and the limiter in its epilogue: tensor-core and
    CUDA-core contractions agree to the FP32 tolerance of the stage increment."""
    cfg = _tc_cfg(name)
    cfg.apply_filter, cfg.pp_limit, cfg.pp_eps = 1, 1, 1e-8
    U = random_state(cfg, 7, amp=0.2)
    gamma = 0.01
    outs = {}
    for tc in (1, 0):
        cfg.mixed_tc = tc
        with FRSolver(cfg) as s:
            d = torch.from_numpy(U).to(cuda)
            out = torch.empty_like(d)
            s.rk_stage_fused(0.0, d, out, A.STAGE_MIXED | A.STAGE_POST_STEP, gamma, a=d, alpha=1.0)
            outs[tc] = out.cpu().numpy()
            rhs = torch.empty_like(d)
            s.rhs_func(0.0, d, rhs)
            scale = float(rhs.abs().max())
            assert s.status() == 0
    # the filter's rows have absolute sums near one; the limiter leaves these states alone
    assert np.max(np.abs(outs[1] - outs[0])) <= 2.0 * TOL_FP32 * gamma * scale


def test_mixed_vortex_with_tensor_cores_matches_fp64_accuracy(cuda):
    """Curved isentropic vortex, p = 4, RK4 to t = 1 with the tensor-core FP32 residual:
    L2 density error within 10 % of the FP64 run's."""
    wl = vortex_curved(n_elems=16, p=4)
    errs = {}
    for mixed in (False, True):
        wl.cfg.mixed_tc = 1
        with FRSolver(wl.cfg) as s:
            x, y = node_coords(wl.cfg, cuda)
            ex = pack2d(*exact_vortex(1.0, x, y))
            J = node_jacobian(wl.cfg, cuda)
            U = wl.init(cuda)
            dt = cfl_time_step(wl.cfg, U, 0.05)
            Integrator(s, "rk4", mixed=mixed).run(U, dt, t_end=1.0)
            errs[mixed] = float(l2_error(wl.cfg, U, ex, J)[0])
            assert s.status() == 0
    assert errs[True] <= 1.1 * errs[False], errs
