"""CPU: the restated oracle pinned to fr_sdg's OWN hot-path code.

Two forms of the pin:
  * fixtures: tests/golden/ref_<case>.npz hold outputs that the reference's
    include/*.hpp (compiled into oracle/_ref/libfrsdg_ref.so by
    oracle/ref_build.py, tests/golden/gen_ref_golden.py) wrote on seeded inputs;
    the oracle must reproduce them.  These tests need nothing but the fixtures.
  * live: when oracle/_ref/libfrsdg_ref.so is built, the oracle and the
    reference library evaluate every parity case of tests/cases.py (p <= 8: the
    reference's GLL class stops at 9 nodes, reference_element.hpp:24,55-59) on the
    same inputs.

Bars: the FP64 forms agree to 1e-12 relative (max|a - b| / max|b|), the
complex-step JVP to the JVP tolerance.  At p <= 3 the two agree bit for bit; above,
the GLL nodes come from different eigen-solvers (the oracle's implicit QL, the
stand-in's Jacobi rotations for Eigen's SelfAdjointEigenSolver) and differ in the
last bits, which moves the residuals by ~1e-15.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests.cases import CASES_1D, CASES_2D, REF_FIXTURES_1D, REF_FIXTURES_2D, _cfg2d, cfg1d, ref_fixture_cfg
from tests.helpers import TOL_FP64, TOL_JVP, cons_to_prim, random_state, rel_err

GOLD = Path(__file__).resolve().parent / "golden"
FIXTURES = list(REF_FIXTURES_2D) + ["1d_" + n for n in REF_FIXTURES_1D]


def _reference():
    from oracle import reference

    if not reference.available():
        pytest.skip("oracle/_ref/libfrsdg_ref.so not built (reference tree absent)")
    return reference


# ---------------------------------------------------------------- fixtures
@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_reproduces_reference_fixture(name):
    d = np.load(GOLD / f"ref_{name}.npz")
    cfg = ref_fixture_cfg(name)
    U, V, Udot = d["U"], d["V"], d["Udot"]
    assert rel_err(O.Oracle(cfg).residual(0.7, U), d["R"]) <= TOL_FP64
    assert rel_err(O.Oracle(cfg).ifunction(0.3, U, Udot), d["IF"]) <= TOL_FP64
    for h, key in ((1e-7, "JV7"), (1e-30, "JV30")):
        cfg.csd_eps = h
        assert rel_err(O.Oracle(cfg).jvp(0.2, 2.5, U, V), d[key]) <= TOL_JVP, key
    cfg.csd_eps = 1e-7
    if cfg.filt_cut_off >= cfg.poly_deg:
        cfg.filt_cut_off = max(cfg.poly_deg - 1, 0)
    for key, (f, w) in (("POSTF", (1, 0)), ("POSTW", (0, 1)), ("POSTB", (1, 1))):
        cfg.apply_filter, cfg.apply_weno, cfg.shock_threshold = f, w, 0.3
        assert rel_err(O.Oracle(cfg).post_step(U), d[key]) <= TOL_FP64, key
    if "P" in d:
        c2 = ref_fixture_cfg(name, cond_sys=True)
        o2 = O.Oracle(c2)
        assert rel_err(o2.prim_to_cons(d["P"]), d["CONS"]) <= TOL_FP64
        assert rel_err(o2.ifunction(0.1, d["P"], Udot), d["IFC"]) <= TOL_FP64
        assert rel_err(o2.jvp(0.1, 1.5, d["P"], V), d["JVC"]) <= TOL_JVP


def test_fixtures_cover_every_output():
    for name in FIXTURES:
        d = np.load(GOLD / f"ref_{name}.npz")
        for key in ("U", "V", "Udot", "R", "IF", "JV7", "JV30", "POSTF", "POSTW", "POSTB"):
            assert key in d and np.all(np.isfinite(d[key])), (name, key)


# ---------------------------------------------------------------- live
def test_fixtures_are_the_reference_outputs():
    """Regenerating the fixtures with the reference library gives the committed files."""
    ref = _reference()
    from tests.golden import gen_ref_golden

    for k, name in enumerate(FIXTURES):
        d = np.load(GOLD / f"ref_{name}.npz")
        fresh = gen_ref_golden.outputs(name, ref.Reference, 500 + k)
        assert sorted(fresh) == sorted(d.files), name
        for key in d.files:
            assert np.array_equal(fresh[key], d[key]), (name, key)


@pytest.mark.parametrize("p", range(1, 9))
def test_reference_element_and_filter(p):
    ref = _reference()
    for c in (0.0, 0.01):
        for a, b in zip(O.reference_element(p, c), ref.reference_element(p, c)):
            assert np.max(np.abs(a - b)) <= 2e-13 * max(1.0, np.max(np.abs(b)))
    if p >= 3:
        assert np.max(np.abs(O.filter_matrix(p) - ref.filter_matrix(p))) <= 1e-14


@pytest.mark.parametrize("name", sorted(n for n in CASES_2D if CASES_2D[n].get("p", 3) <= 8))
def test_oracle_vs_reference_2d(name):
    ref = _reference()
    cfg = _cfg2d(**CASES_2D[name])
    U = random_state(cfg, seed=17)
    Us = random_state(cfg, seed=18, smooth=True)
    rng = np.random.default_rng(19)
    V, Udot = rng.normal(size=U.size), rng.normal(size=U.size)
    o, r = O.Oracle(cfg, threads=4), ref.Reference(cfg)
    assert rel_err(o.residual(0.4, U), r.residual(0.4, U)) <= TOL_FP64
    assert rel_err(o.rhs(0.4, Us), r.rhs(0.4, Us)) <= TOL_FP64
    assert rel_err(o.ifunction(0.4, U, Udot), r.ifunction(0.4, U, Udot)) <= TOL_FP64
    Uc = U.astype(np.complex128) + 1e-3j * V
    assert rel_err(o.residual_complex(0.4, Uc).view(np.float64), r.residual_complex(0.4, Uc).view(np.float64)) \
        <= TOL_FP64
    for h in (1e-7, 1e-30):
        cfg.csd_eps = h
        assert rel_err(O.Oracle(cfg).jvp(0.4, 1.7, U, V), ref.Reference(cfg).jvp(0.4, 1.7, U, V)) <= TOL_JVP


@pytest.mark.parametrize("stab", ["filter", "weno", "both"])
@pytest.mark.parametrize("name", ["cart_ideal_rusanov_p3", "cart_vdw_rusanov_p5_perx", "sinewarp_hllc_p4_periodic",
                                  "cart_ideal_hllc_p7", "cart_vdw_hllc_p8_periodic", "wedge_bc_hllc_p3"])
def test_oracle_vs_reference_post_step_2d(name, stab):
    ref = _reference()
    kw = dict(CASES_2D[name])
    kw.update(apply_filter=stab in ("filter", "both"), apply_weno=stab in ("weno", "both"), threshold=0.3)
    cfg = _cfg2d(**kw)
    U = random_state(cfg, seed=31)
    assert rel_err(O.Oracle(cfg).post_step(U), ref.Reference(cfg).post_step(U)) <= TOL_FP64


@pytest.mark.parametrize("name", ["cart_ideal_hllc_p2", "sinewarp_hllc_p4_periodic", "cart_vdw_hllc_p4_walls",
                                  "bump_hllc_p3_inflow_outlet"])
def test_oracle_vs_reference_change_of_variables(name):
    ref = _reference()
    cfg = _cfg2d(**CASES_2D[name])
    cfg.cond_sys = 1
    P = cons_to_prim(cfg, random_state(cfg, seed=21, smooth=True))
    rng = np.random.default_rng(22)
    Udot, V = rng.normal(size=P.size), rng.normal(size=P.size)
    o, r = O.Oracle(cfg), ref.Reference(cfg)
    assert rel_err(o.prim_to_cons(P), r.prim_to_cons(P)) <= TOL_FP64
    assert rel_err(o.ifunction(0.1, P, Udot), r.ifunction(0.1, P, Udot)) <= TOL_FP64
    assert rel_err(o.jvp(0.1, 1.5, P, V), r.jvp(0.1, 1.5, P, V)) <= TOL_JVP


@pytest.mark.parametrize("name", sorted(n for n in CASES_1D if CASES_1D[n].get("p", 3) <= 8))
def test_oracle_vs_reference_1d(name):
    ref = _reference()
    cfg = cfg1d(name)
    U = random_state(cfg, seed=41)
    rng = np.random.default_rng(42)
    V, Udot = rng.normal(size=U.size), rng.normal(size=U.size)
    o, r = O.Oracle(cfg), ref.Reference(cfg)
    assert rel_err(o.residual(0.0, U), r.residual(0.0, U)) <= TOL_FP64
    assert rel_err(o.ifunction(0.0, U, Udot), r.ifunction(0.0, U, Udot)) <= TOL_FP64
    assert rel_err(o.jvp(0.0, 3.0, U, V), r.jvp(0.0, 3.0, U, V)) <= TOL_JVP
    for stab in ("filter", "weno"):
        c = cfg1d(name, apply_filter=stab == "filter", apply_weno=stab == "weno", threshold=0.3)
        if c.apply_filter and c.filt_cut_off >= c.poly_deg:
            c.filt_cut_off = c.poly_deg - 1
        assert rel_err(O.Oracle(c).post_step(U), ref.Reference(c).post_step(U)) <= TOL_FP64, stab
    cfg.cond_sys = 1
    Us = random_state(cfg, seed=43, smooth=True)
    P = cons_to_prim(cfg, Us)
    assert rel_err(O.Oracle(cfg).prim_to_cons(P), ref.Reference(cfg).prim_to_cons(P)) <= TOL_FP64


@pytest.mark.parametrize("threads", [2, 3, 5])
def test_reference_threaded_rhs_is_the_single_thread_rhs(threads):
    """The reference arm's host-thread form (one block of element rows per thread, as
    MPI ranks) computes the same numbers as the one-rank residual."""
    ref = _reference()
    for name in ("cart_vdw_rusanov_p5_perx", "vortex_dirichlet_p3", "bump_hllc_p3_inflow_outlet"):
        cfg = _cfg2d(**CASES_2D[name])
        U = random_state(cfg, seed=3)
        one = ref.Reference(cfg).rhs(0.1, U)
        many = ref.Reference(cfg, threads=threads).rhs(0.1, U)
        assert np.array_equal(one, many), name
        assert np.array_equal(ref.Reference(cfg, threads=threads).residual(0.1, U), -one), name


def test_reference_default_config_is_the_library_default():
    """The reference arm builds its configuration without the CUDA library; its
    defaults equal frsdg_config_default field by field."""
    import ctypes

    from fr_sdg_b200 import _abi as A
    from oracle import reference

    a, b = A.frsdg_config(), A.frsdg_config()
    A.check(A.lib().frsdg_config_default(a), "frsdg_config_default")
    reference.default_config(b)
    assert ctypes.string_at(ctypes.addressof(a), ctypes.sizeof(a)) == ctypes.string_at(ctypes.addressof(b),
                                                                                           ctypes.sizeof(b))
