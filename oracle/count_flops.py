"""Count the floating-point operations of one residual of the benchmark workload with
the oracle's counting scalar (flop_count.cpp) and write profiles/fr2d_kernel_blast_flops.txt.

Measurement infrastructure (run here, not on the GPU): the count is that of the
reference's algorithm as restated by the oracle, one operation per +, -, *, / and
square root.  Operations per element are fitted as a M^2 + b M on M x M meshes of the
workload (b carries the boundary faces) and evaluated at the benchmark's 1024^2.

    python oracle/count_flops.py
"""
from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
# run as a script, this directory comes first on the path and its oracle.py would
# shadow the oracle package
sys.path = [str(ROOT)] + [q for q in sys.path if Path(q or ".").resolve() != Path(__file__).resolve().parent]

from fr_sdg_b200.workloads import blast_large  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

OUT = ROOT / "profiles" / "fr2d_kernel_blast_flops.txt"


def count(m: int, p: int = 5) -> dict:
    wl = blast_large(n_elems=m, p=p)
    o = Oracle(wl.cfg)
    return o.count_flops(0.0, wl.init("cpu").numpy())


def main() -> None:
    sizes = (16, 32)
    c = {m: count(m) for m in sizes}
    tot = {m: sum(v for k, v in c[m].items() if k != "other") for m in sizes}
    m1, m2 = sizes
    # tot = a m^2 + b m
    b = (tot[m2] - tot[m1] * (m2 / m1) ** 2) / (m2 - m2 * m2 / m1)
    a = (tot[m1] - b * m1) / m1 ** 2
    full = a * 1024 ** 2 + b * 1024
    nodes = 1024 ** 2 * 36
    lines = [
        "Residual of the blast workload (2D, p = 5, HLLC, Van der Waals) -- operation count of one",
        "residual evaluation by the oracle's counting scalar (one per +, -, *, /, sqrt; no FMA credit)",
        "",
        "    python oracle/count_flops.py",
        "",
    ]
    for m in sizes:
        lines.append(f"{m}x{m} elements: " + ", ".join(f"{k} {v}" for k, v in c[m].items()) + f"; total {tot[m]}")
    lines += [
        "",
        f"fit: ops = {a:.1f} M^2 + {b:.1f} M  ({a:.1f} per element, {a / 36:.1f} per node)",
        f"flops_per_full_launch: {int(round(full))}",
        f"(1024^2 elements, {nodes} nodes; {full / (2 * 8 * nodes * 4):.2f} flop per algorithmic byte)",
    ]
    OUT.write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
