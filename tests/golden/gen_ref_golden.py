"""Generate tests/golden/ref_<case>.npz: outputs of fr_sdg's OWN hot-path code
(the reference's include/*.hpp compiled into oracle/_ref/libfrsdg_ref.so by
oracle/ref_build.py) on seeded inputs of the cases in tests/cases.py
(REF_FIXTURES_2D, REF_FIXTURES_1D).  These fixtures pin the restated oracle and
the CUDA library to the reference itself.

Per case: U (seeded state), V (seeded direction), Udot, and
  R     = residual_kernel(U) at t = 0.7
  IF    = fun_implicit: Udot + R(U) at t = 0.3
  JV7   = complex-step matmult at (t 0.2, sigma 2.5), h = 1e-7 (the reference's)
  JV30  = the same with h = 1e-30
  POSTF = apply_stabilization with the spectral filter (threshold 0.3)
  POSTW = the same with WENO + shock sensor
  POSTB = both (the reference then keeps the filter's result)
and, for the change-of-variables cases (2D names ending in _cond), P (primitive
state), CONS = primitive_to_conservative(P), IFC and JVC (ifunction and JVP with
cond_sys on).

    python tests/golden/gen_ref_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

COND_CASES = ("cart_vdw_hllc_p4_walls", "sinewarp_hllc_p4_periodic")


def outputs(name: str, ref_cls, seed: int) -> dict:
    from tests.cases import ref_fixture_cfg
    from tests.helpers import cons_to_prim, random_state

    cfg = ref_fixture_cfg(name)
    U = random_state(cfg, seed=seed)
    rng = np.random.default_rng(seed + 1)
    V = rng.normal(size=U.size)
    Udot = rng.normal(size=U.size)
    out = {"U": U, "V": V, "Udot": Udot}
    r = ref_cls(cfg)
    out["R"] = r.residual(0.7, U)
    out["IF"] = r.ifunction(0.3, U, Udot)
    for h, key in ((1e-7, "JV7"), (1e-30, "JV30")):
        cfg.csd_eps = h
        out[key] = ref_cls(cfg).jvp(0.2, 2.5, U, V)
    cfg.csd_eps = 1e-7
    if cfg.filt_cut_off >= cfg.poly_deg:
        cfg.filt_cut_off = max(cfg.poly_deg - 1, 0)
    for key, (f, w) in (("POSTF", (1, 0)), ("POSTW", (0, 1)), ("POSTB", (1, 1))):
        cfg.apply_filter, cfg.apply_weno, cfg.shock_threshold = f, w, 0.3
        out[key] = ref_cls(cfg).post_step(U)
    if name in COND_CASES:
        c2 = ref_fixture_cfg(name, cond_sys=True)
        Us = random_state(c2, seed=seed + 2, smooth=True)
        P = cons_to_prim(c2, Us)
        r2 = ref_cls(c2)
        out["P"] = P
        out["CONS"] = r2.prim_to_cons(P)
        out["IFC"] = r2.ifunction(0.1, P, Udot)
        out["JVC"] = r2.jvp(0.1, 1.5, P, V)
    return out


def main() -> None:
    from oracle.reference import Reference
    from tests.cases import REF_FIXTURES_1D, REF_FIXTURES_2D

    names = list(REF_FIXTURES_2D) + ["1d_" + n for n in REF_FIXTURES_1D]
    for k, name in enumerate(names):
        np.savez_compressed(HERE / f"ref_{name}.npz", **outputs(name, Reference, 500 + k))
        print("wrote", f"ref_{name}.npz")


if __name__ == "__main__":
    main()
