"""Recipe for oracle/_ref/libfrsdg_ref.so: fr_sdg's own hot-path headers compiled
into a CPU library, the checker that pins the restated oracle.

TEST INFRASTRUCTURE ONLY.  The reference needs PETSc, Eigen, Boost.Math and gcc >= 14
(<print>, C++23/26 relaxations); none is in this image.  The recipe therefore
  * compiles oracle/ref_capi.cpp against the stand-ins in oracle/ref_shim (a one-rank
    PETSc DMDA, the Eigen dense subset, Legendre recurrences for Boost.Math, <print>
    on <format>);
  * reads the reference's include/*.hpp where they lie; the two headers that
    gcc 13 rejects are rewritten into a temporary directory (never into this
    repository) with each change applied to exactly one known line:
      physics_impl_2D.hpp:274  `constexpr auto n_eqs = this->get_n_eqs();`
          gcc 13 does not allow `this` in a constant expression (P2280, gcc 14);
          rewritten as `constexpr std::size_t n_eqs = 4;` (get_n_eqs() returns 4);
      physics_evaluator.hpp:194-195  `m_stab{.x{...}, .y{...}}`
          gcc 13 rejects an explicit constructor in a designated braced member
          initialiser; rewritten as `.x = StabilizationTechniques<T>(...)` (same
          constructor, same arguments).
The output is only oracle/_ref/libfrsdg_ref.so.

    python oracle/ref_build.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libfrsdg_ref.so"
DEFAULT_REFERENCE = Path(os.environ.get("FRSDG_REFERENCE", "/root/reference"))

# (header, original text, replacement): each original must occur exactly once
REWRITES = [
    ("physics_impl_2D.hpp",
     "constexpr auto n_eqs = this->get_n_eqs();",
     "constexpr std::size_t n_eqs = 4; /* gcc 13: was this->get_n_eqs() */"),
    ("physics_evaluator.hpp",
     "m_stab{.x{m_gll_x, m_opts, m_cached_data_x, 0},",
     "m_stab{.x = StabilizationTechniques<T>(m_gll_x, m_opts, m_cached_data_x, 0),"),
    ("physics_evaluator.hpp",
     ".y{m_gll_y, m_opts, m_cached_data_y, 1}},",
     ".y = StabilizationTechniques<T>(m_gll_y, m_opts, m_cached_data_y, 1)},"),
]


def available(reference: Path = DEFAULT_REFERENCE) -> bool:
    return (reference / "include" / "physics_evaluator.hpp").exists()


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False, verbose: bool = False) -> Path | None:
    """Build the library when the reference tree is present; returns its path, or
    None when neither the reference nor a previously built library exists."""
    if not available(reference):
        return LIB if LIB.exists() else None
    srcs = [HERE / "ref_capi.cpp", *sorted((HERE / "ref_shim").rglob("*")), HERE / "ref_build.py",
            HERE.parent / "include" / "frsdg.h"]
    inc = reference / "include"
    newest = max([p.stat().st_mtime for p in srcs if p.is_file()] + [p.stat().st_mtime for p in inc.glob("*.hpp")])
    if not force and LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="frsdg_ref_") as tmp:
        compat = Path(tmp) / "include"
        compat.mkdir()
        # the reference's headers include each other by name from their own directory,
        # so the directory is mirrored: every header a symlink, except the rewritten ones
        rewritten = {name for name, _, _ in REWRITES}
        for h in inc.iterdir():
            if h.name not in rewritten:
                os.symlink(h, compat / h.name)
        for name in rewritten:
            text = (inc / name).read_text()
            for hdr, old, new in REWRITES:
                if hdr != name:
                    continue
                if text.count(old) != 1:
                    raise RuntimeError(f"{name}: expected exactly one occurrence of {old!r}")
                text = text.replace(old, new)
            (compat / name).write_text(text)
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++23", "-O2", "-fPIC", "-shared", "-w",
               "-I", str(HERE / "ref_shim"), "-I", str(compat),
               str(HERE / "ref_capi.cpp"), "-o", str(LIB.with_suffix(".so.tmp"))]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"reference build failed:\n{res.stderr[-4000:]}")
        os.replace(LIB.with_suffix(".so.tmp"), LIB)
    if verbose:
        print(f"built {LIB}", flush=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    out = build(a.reference, a.force, verbose=True)
    if out is None:
        print(f"reference tree not found at {a.reference}; nothing built")
    return 0


if __name__ == "__main__":
    sys.exit(main())
