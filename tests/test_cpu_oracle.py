"""CPU: the oracle and the library's host set-up against the reference's known
answers (tests/sbp.cpp, tests/filter_check.cpp, reference_element.hpp:41-45,
factory.hpp:33-56) and the committed golden fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

import fr_sdg_b200 as F
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config
from oracle import oracle as O
from tests.helpers import random_state, rel_err

GOLD = Path(__file__).resolve().parent / "golden"
PS = range(1, 10)


@pytest.fixture(scope="module")
def gll_gold():
    return json.loads((GOLD / "gll_tables.json").read_text())


@pytest.mark.parametrize("p", PS)
@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_gll_nodes_weights_vs_golden(p, impl, gll_gold):
    x, w = (O.reference_element(p) if impl == "oracle" else F.reference_element(p))[:2]
    g = gll_gold[str(p)]
    assert np.max(np.abs(x - np.array(g["nodes"]))) <= 4e-16
    assert np.max(np.abs(w - np.array(g["weights"]))) <= 2e-15
    assert abs(w.sum() - 2.0) <= 1e-14  # reference_element.hpp:41-45


def test_gll_closed_forms():
    for impl in (O.reference_element, F.reference_element):
        assert np.allclose(impl(2)[0], [-1, 0, 1], atol=1e-16)
        assert np.allclose(impl(3)[0], [-1, -1 / np.sqrt(5), 1 / np.sqrt(5), 1], atol=2e-16)
        assert np.allclose(impl(4)[0], [-1, -np.sqrt(3 / 7), 0, np.sqrt(3 / 7), 1], atol=2e-16)


@pytest.mark.parametrize("p", PS)
@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_sbp_identity(p, impl):
    """tests/sbp.cpp:9-51: M D + D^T M = diag(-1, 0, ..., 0, 1)."""
    x, w, D, _, _ = O.reference_element(p) if impl == "oracle" else F.reference_element(p)
    n = p + 1
    Q = np.diag(w) @ D
    B = np.zeros((n, n))
    B[0, 0], B[-1, -1] = -1.0, 1.0
    assert np.linalg.norm(Q + Q.T - B) <= 5e-14


@pytest.mark.parametrize("p", PS)
def test_differentiation_exact_on_polynomials(p):
    x, _, D, _, _ = F.reference_element(p)
    for k in range(p + 1):
        d = D @ x ** k
        exact = k * x ** (k - 1) if k > 0 else np.zeros_like(x)
        assert np.max(np.abs(d - exact)) <= 1e-12 * max(1, k * k)


@pytest.mark.parametrize("p", range(3, 10))
@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_filter_eigenvalues_are_sigma(p, impl):
    """tests/filter_check.cpp:14-39: the filter's eigenvalues are the sigma_i."""
    Fm = (O.filter_matrix if impl == "oracle" else F.filter_matrix)(p, 2, 32, 36.0)
    n = p + 1
    sig = [1.0 if i < 2 else np.exp(-36.0 * ((i - 2) / (n - 1 - 2)) ** 32) for i in range(n)]
    ev = np.sort(np.linalg.eigvals(Fm).real)
    assert np.max(np.abs(ev - np.sort(sig))) <= 1e-12


@pytest.mark.parametrize("p", PS)
def test_library_setup_matches_oracle(p):
    for c in (0.0, 0.01):
        a = O.reference_element(p, c)
        b = F.reference_element(p, c)
        for u, v in zip(a, b):
            assert np.max(np.abs(u - v)) <= 5e-14 * max(1.0, np.max(np.abs(u)))
    if p >= 3:
        assert np.max(np.abs(O.filter_matrix(p) - F.filter_matrix(p))) <= 1e-14


@pytest.mark.parametrize("p", PS)
def test_vcjh_dg_correction(p):
    """c = 0: g_R is the right Radau polynomial, g_R'(1) = (p+1)^2/2 and g_L' mirrors g_R'."""
    x, _, _, dL, dR = F.reference_element(p, 0.0)
    assert abs(dR[-1] - (p + 1) ** 2 / 2.0) <= 1e-12 * (p + 1) ** 2
    assert np.max(np.abs(dL + dR[::-1])) <= 1e-12 * (p + 1) ** 2


def _const_state(cfg, q):
    n = cfg.poly_deg + 1
    if cfg.dim == 2:
        return np.tile(np.array(q, dtype=float), cfg.n_elems[0] * cfg.n_elems[1] * n * n)
    return np.tile(np.repeat(np.array(q, dtype=float), n), cfg.n_elems[0])


@pytest.mark.parametrize("geom", [A.GEOM_CARTESIAN, A.GEOM_SINE_WARP, A.GEOM_DELAVAL])
@pytest.mark.parametrize("riemann", ["rusanov", "hllc"])
def test_oracle_free_stream(geom, riemann):
    """DoNothing (factory.hpp:33-56): a constant state on a periodic mesh has R = 0."""
    per = {f: A.BC_PERIODIC for f in range(4)}
    cfg = make_config(dim=2, p=4, n_elems=(5, 4), box=(10.0, 10.0), riemann=riemann, geometry=geom,
                      geom_params=(0.1, 0, 0, 0), bcs=per)
    R = O.Oracle(cfg).residual(0.0, _const_state(cfg, [1.0, 2.0, 3.0, 9.0]))
    assert np.max(np.abs(R)) <= 1e-11  # fluxes O(10), metric terms O(1): rounding only
    cfg1 = make_config(dim=1, p=3, n_elems=(8, 1), riemann=riemann, bcs={A.LEFT: A.BC_PERIODIC, A.RIGHT: A.BC_PERIODIC})
    R1 = O.Oracle(cfg1).residual(0.0, _const_state(cfg1, [1.0, 2.0, 3.0]))
    assert np.max(np.abs(R1)) <= 1e-12


@pytest.mark.parametrize("name", ["cart_vdw_hllc_p3", "sinewarp_rusanov_p4", "sod1d_rusanov_p3"])
def test_oracle_against_golden(name):
    from tests.golden import gen_golden  # noqa: F401  (documents the generator)

    d = np.load(GOLD / f"residual_{name}.npz")
    cfgs = {
        "cart_vdw_hllc_p3": make_config(dim=2, p=3, n_elems=(5, 4), box=(1.0, 0.8), riemann="hllc", gas="vdw",
                                        vdw=(0.05, 0.02),
                                        bcs={A.LEFT: A.BC_WALL, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_WALL,
                                             A.BOTTOM: A.BC_OUTFLOW}, apply_filter=True),
        "sinewarp_rusanov_p4": make_config(dim=2, p=4, n_elems=(4, 4), box=(10.0, 10.0), riemann="rusanov",
                                           geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                           bcs={f: A.BC_PERIODIC for f in range(4)}, apply_filter=True),
        "sod1d_rusanov_p3": make_config(dim=1, p=3, n_elems=(20, 1), riemann="rusanov",
                                        bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW}, apply_filter=True),
    }
    o = O.Oracle(cfgs[name])
    assert rel_err(o.residual(0.5, d["U"]), d["R"]) <= 1e-14
    assert rel_err(o.jvp(0.5, 2.0, d["U"], d["V"]), d["JV"]) <= 1e-14
    assert rel_err(o.post_step(d["U"]), d["POST"]) <= 1e-14


def test_oracle_jvp_is_a_derivative():
    """The complex-step JVP (h = 1e-30) matches a central finite difference of R."""
    cfg = make_config(dim=2, p=3, n_elems=(4, 4), riemann="hllc", gas="vdw", vdw=(0.05, 0.02),
                      bcs={A.LEFT: A.BC_WALL, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_OUTFLOW, A.BOTTOM: A.BC_WALL},
                      csd_eps=1e-30)
    U = random_state(cfg, seed=3, smooth=True)
    V = np.random.default_rng(4).normal(size=U.size)
    o = O.Oracle(cfg)
    jv = o.jvp(0.0, 0.0, U, V)
    eps = 1e-6
    fd = (o.residual(0.0, U + eps * V) - o.residual(0.0, U - eps * V)) / (2 * eps)
    assert rel_err(jv, fd) <= 1e-6


def test_oracle_complex_residual_real_part():
    cfg = make_config(dim=2, p=2, n_elems=(4, 3), riemann="hllc")
    U = random_state(cfg, seed=8)
    o = O.Oracle(cfg)
    Rc = o.residual_complex(0.0, U.astype(np.complex128))
    assert np.array_equal(Rc.real, o.residual(0.0, U))
    assert np.all(Rc.imag == 0.0)


def test_flop_count_scales_with_elements():
    """The oracle's counting scalar: a residual's operation count is deterministic and
    grows as a M^2 + b M on M x M meshes (interior plus boundary faces)."""
    from fr_sdg_b200.workloads import blast_large
    from oracle.oracle import Oracle

    counts = {}
    for m in (4, 8, 16):
        wl = blast_large(n_elems=m, p=2)
        U = wl.init("cpu").numpy()
        c1 = Oracle(wl.cfg).count_flops(0.0, U)
        c2 = Oracle(wl.cfg).count_flops(0.0, U)
        assert c1 == c2 and c1["add"] > 0 and c1["sqrt"] > 0 and c1["other"] == 0
        counts[m] = sum(c1.values())
    b = (counts[8] - 4 * counts[4]) / (8 - 16)
    a = (counts[4] - 4 * b) / 16
    assert abs(a * 256 + b * 16 - counts[16]) <= 1e-9 * counts[16]
