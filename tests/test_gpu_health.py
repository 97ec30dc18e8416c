"""GPU: failure detection without a GPU fault -- the device health word counts exactly
the nodes a host-injected state poisons (NaN or non-positive density), frsdg_check_state
covers states no residual has read, the integrator rejects and retakes failed steps
with halved dt -- and the library's FP64 reciprocal and square root against IEEE
division and sqrt."""
import math

import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from tests.cases import CASES_2D, _cfg2d, cfg1d
from tests.helpers import random_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cart_vdw_hllc_p4_walls", "sinewarp_hllc_p4_periodic", "cart_ideal_hllc_p7"])
def test_health_word_counts_poisoned_nodes_2d(name, cuda):
    cfg = _cfg2d(**CASES_2D[name])
    U = random_state(cfg, seed=21)
    nodes = U.size // 4
    rng = np.random.default_rng(22)
    pick = rng.choice(nodes, size=23, replace=False)
    bad_vals = [np.nan, -1.0, 0.0, -np.inf, np.inf]
    for k, q in enumerate(pick):
        U[4 * q] = bad_vals[k % len(bad_vals)]
    with FRSolver(cfg) as s:
        Ud = torch.from_numpy(U).to(cuda)
        R = torch.empty_like(Ud)
        assert s.status() == 0
        s.residual_kernel(0.0, Ud, R)
        assert s.status() == len(pick)  # every poisoned node counted once
        assert s.status() == 0          # and the word restarts at zero
        s.check_state(Ud)
        assert s.status() == len(pick)
        s.rhs_func(0.0, Ud, R)
        s.check_state(Ud)
        assert s.status() == 2 * len(pick)


def test_health_word_counts_poisoned_nodes_1d(cuda):
    cfg = cfg1d("vdw_hllc_p5_walls")
    U = random_state(cfg, seed=23)
    n = cfg.poly_deg + 1
    elems = [0, 5, 17, cfg.n_elems[0] - 1]
    for e in elems:
        U[e * 3 * n + (e % n)] = np.nan if e % 2 else -0.5
    with FRSolver(cfg) as s:
        Ud = torch.from_numpy(U).to(cuda)
        s.check_state(Ud)
        assert s.status() == len(elems)


def test_step_rejection_on_the_gpu(cuda):
    """Circular explosion, p = 2, WENO + shock sensor, no positivity limiter, CFL 0.1
    (dt = 0.1 h / c_max): the first step loses positivity (as fr_sdg's own code does);
    with rejection the failed steps are retaken as half steps and the run stays finite."""
    from fr_sdg_b200.integrate import Integrator, cfl_time_step
    from fr_sdg_b200.workloads import circular_explosion

    wl = circular_explosion(32, 2, "ideal", 1.4, (0.0, 0.0), 0.4, 0.1, filt_cut_off=1)
    cfg = wl.cfg
    cfg.apply_filter, cfg.apply_weno, cfg.pp_limit = 0, 1, 0
    with FRSolver(cfg) as s:
        U0 = wl.init(cuda)
        dt = cfl_time_step(cfg, U0, 0.1)
        U = U0.clone()
        Integrator(s, "ssprk3").step(U, 0.0, dt)
        s.check_state(U)
        Integrator(s, "ssprk3").step(U, dt, dt)
        assert s.status() > 0  # the plain run goes bad
        U = U0.clone()
        st = Integrator(s, "ssprk3").run(U, dt, t_end=8 * dt, max_reject=4)
        assert st.rejected >= 1 and abs(st.t - 8 * dt) < 1e-15
        assert bool(torch.isfinite(U).all()) and float(U.view(-1, 4)[:, 0].min()) > 0.0


def _ulps(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Distance in units in the last place of finite doubles of the same sign."""
    ia, ib = a.view(torch.int64), b.view(torch.int64)
    return (ia - ib).abs()


@pytest.mark.parametrize("op", ["rcp", "sqrt"])
def test_device_reciprocal_and_sqrt_within_two_ulp(op, cuda):
    g = torch.Generator(device="cpu").manual_seed(24)
    exps = torch.randint(-300, 300, (1_000_000,), generator=g).to(torch.float64)
    mant = 1.0 + torch.rand(1_000_000, generator=g, dtype=torch.float64)
    x = mant * torch.pow(2.0, exps)
    if op == "rcp":
        x = torch.where(torch.rand(1_000_000, generator=g) < 0.5, x, -x)
    edge = torch.tensor([1.0, 2.0, 0.5, 3.0, 1e-37, 1e37, 1.1e-37, 0.9e37, 1e-300, 1e300, 2.2250738585072014e-308,
                         4.9e-324, 1e-310, 1.7976931348623157e308, 0.0, -0.0, float("inf"), -float("inf"),
                         float("nan"), -1.0, -1e-200,
                         # the edges of the fast paths' range [2^-122, 2^123)
                         2.0 ** -122, math.nextafter(2.0 ** -122, 0.0), 2.0 ** 123, math.nextafter(2.0 ** 123, 0.0),
                         -2.0 ** -122, -math.nextafter(2.0 ** 123, 0.0)], dtype=torch.float64)
    x = torch.cat([x, edge]).to(cuda)
    y = torch.empty_like(x)
    A.check(A.lib().frsdg_device_math(0 if op == "rcp" else 1, x.data_ptr(), y.data_ptr(), x.numel(), None),
            "frsdg_device_math")
    # the deferred form of the residual's passes equals the checked function bit for bit
    yd = torch.empty_like(x)
    A.check(A.lib().frsdg_device_math(2 if op == "rcp" else 3, x.data_ptr(), yd.data_ptr(), x.numel(), None),
            "frsdg_device_math")
    torch.cuda.synchronize()
    assert torch.equal(torch.isnan(yd), torch.isnan(y))
    assert torch.equal(yd[~torch.isnan(y)], y[~torch.isnan(y)])
    ref = 1.0 / x if op == "rcp" else torch.sqrt(x)
    fin = torch.isfinite(ref) & (ref != 0)
    assert torch.equal(torch.isnan(y), torch.isnan(ref))
    assert torch.equal(y[~fin & ~torch.isnan(ref)], ref[~fin & ~torch.isnan(ref)])  # +-inf and +-0 alike
    assert int(_ulps(y[fin], ref[fin]).max()) <= 2


@pytest.mark.parametrize("op", ["rcp", "sqrt"])
def test_fp32_fast_reciprocal_and_sqrt_within_two_ulp(op, cuda):
    """The FP32 reciprocal and square root of the mixed residual (hardware approximation
    plus one Newton step, IEEE operations outside [2^-125, 2^125)) against IEEE float
    division and sqrt: within 2 float ulps, zeros, infinities and NaNs alike."""
    g = torch.Generator(device="cpu").manual_seed(25)
    exps = torch.randint(-140, 128, (1_000_000,), generator=g).to(torch.float64)
    mant = 1.0 + torch.rand(1_000_000, generator=g, dtype=torch.float64)
    xf = (mant * torch.pow(2.0, exps)).float()
    if op == "rcp":
        xf = torch.where(torch.rand(1_000_000, generator=g) < 0.5, xf, -xf)
    edge = torch.tensor([1.0, 2.0, 0.5, 3.0, 2.0 ** -125, 2.0 ** 125, 2.0 ** 124, 1e-45, 1e-40, 3.4e38, 0.0, -0.0,
                         float("inf"), -float("inf"), float("nan"), -1.0], dtype=torch.float32)
    xf = torch.cat([xf, edge])
    x = xf.double().to(cuda)
    y = torch.empty_like(x)
    A.check(A.lib().frsdg_device_math(4 if op == "rcp" else 5, x.data_ptr(), y.data_ptr(), x.numel(), None),
            "frsdg_device_math")
    torch.cuda.synchronize()
    got = y.float().cpu()
    ref = 1.0 / xf if op == "rcp" else torch.sqrt(xf)
    assert torch.equal(torch.isnan(got), torch.isnan(ref))
    fin = torch.isfinite(ref) & (ref != 0) & (ref.abs() >= torch.finfo(torch.float32).tiny)
    other = ~fin & ~torch.isnan(ref)
    assert torch.equal(got[other & ((ref == 0) | torch.isinf(ref))], ref[other & ((ref == 0) | torch.isinf(ref))])
    ulps = (got[fin].view(torch.int32).long() - ref[fin].view(torch.int32).long()).abs()
    assert int(ulps.max()) <= 2
