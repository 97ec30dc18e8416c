"""Generate the golden fixtures of tests/golden/.

* gll_tables.json -- GLL nodes and weights for p = 1..9 computed independently
  of both the oracle and the library: the interior nodes are the roots of
  P'_p found by numpy.polynomial.legendre (companion-matrix eigenvalues) and
  polished by Newton in numpy's longdouble; weights 2 / (p (p+1) P_p(x)^2).
  These are the closed-form tables the reference's GLL class
  (reference_element.hpp:50-147) must reproduce, and the weights sum to 2
  (reference_element.hpp:41-45).
* residual_*.npz -- seeded input states and the oracle's residual / JVP / post-step
  outputs on small meshes, pinning the oracle against drift.

    python tests/golden/gen_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
from numpy.polynomial import legendre as L

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def gll_table(p: int):
    cp = np.zeros(p + 1)
    cp[p] = 1.0
    dcp = L.legder(cp)
    inner = np.sort(L.legroots(dcp).real) if p >= 2 else np.array([])
    # Newton polish on P'_p in long double
    x = inner.astype(np.longdouble)
    for _ in range(5):
        f = np.array([L.legval(float(v), dcp) for v in x], dtype=np.longdouble)
        df = np.array([L.legval(float(v), L.legder(dcp)) for v in x], dtype=np.longdouble)
        x = x - f / df if len(x) else x
    nodes = np.concatenate([[-1.0], np.asarray(x, dtype=np.float64), [1.0]])
    Pp = L.legval(nodes, cp)
    w = 2.0 / (p * (p + 1) * Pp * Pp)
    return nodes, w


def main():
    tables = {}
    for p in range(1, 10):
        x, w = gll_table(p)
        tables[str(p)] = {"nodes": x.tolist(), "weights": w.tolist()}
    (HERE / "gll_tables.json").write_text(json.dumps(tables, indent=1))

    from fr_sdg_b200 import _abi as A
    from fr_sdg_b200.workloads import make_config
    from oracle.oracle import Oracle
    from tests.helpers import random_state

    cases = {
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
    for name, cfg in cases.items():
        U = random_state(cfg, seed=1234)
        V = np.random.default_rng(99).normal(size=U.size)
        o = Oracle(cfg)
        np.savez_compressed(HERE / f"residual_{name}.npz", U=U, V=V, R=o.residual(0.5, U),
                            JV=o.jvp(0.5, 2.0, U, V), POST=o.post_step(U))


if __name__ == "__main__":
    main()
