"""Parity cases shared by the CPU pin tests and the GPU parity tests: seeded
configurations covering p = 1..9, both gases, both Riemann solvers, every geometry
policy and every boundary kind (2D), and the 1D variants (radial source, Dirichlet,
walls, periodic)."""
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.workloads import make_config

PER = (A.BC_PERIODIC, None, None)
OUT = A.BC_OUTFLOW


def _cfg2d(**kw):
    base = dict(dim=2, p=3, n_elems=(7, 5), box=(1.3, 0.9), riemann="hllc",
                bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: OUT, A.BOTTOM: OUT})
    base.update(kw)
    return make_config(**base)


VDW = dict(gas="vdw", vdw=(0.05, 0.02))
VORTEX = (A.BC_VORTEX, None, (1.0, 1.0, 5.0, 1.0, 10.0))

CASES_2D = {
    "cart_ideal_rusanov_p3": dict(riemann="rusanov"),
    "cart_ideal_hllc_p1_periodic": dict(p=1, n_elems=(9, 6), bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "cart_ideal_hllc_p2": dict(p=2, n_elems=(11, 9)),
    "cart_vdw_hllc_p4_walls": dict(p=4, **VDW, bcs={A.LEFT: A.BC_WALL, A.RIGHT: OUT, A.TOP: A.BC_WALL, A.BOTTOM: OUT}),
    "cart_vdw_rusanov_p5_perx": dict(p=5, riemann="rusanov", **VDW,
                                     bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: A.BC_WALL, A.BOTTOM: A.BC_WALL}),
    "cart_ideal_hllc_p6": dict(p=6, n_elems=(5, 5), radau_corr=0.01),
    "cart_ideal_hllc_p7": dict(p=7, n_elems=(3, 5)),
    "cart_vdw_hllc_p8_periodic": dict(p=8, n_elems=(4, 3), **VDW, bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "cart_ideal_rusanov_p9": dict(p=9, n_elems=(3, 2), riemann="rusanov"),
    "sinewarp_hllc_p4_periodic": dict(p=4, n_elems=(6, 6), box=(10.0, 10.0), geometry=A.GEOM_SINE_WARP,
                                      geom_params=(0.1, 0, 0, 0),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "sinewarp_vdw_rusanov_p3": dict(p=3, n_elems=(5, 7), box=(2.0, 3.0), geometry=A.GEOM_SINE_WARP,
                                    geom_params=(0.05, 0, 0, 0), riemann="rusanov", **VDW,
                                    bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: A.BC_WALL, A.BOTTOM: OUT}),
    "bump_hllc_p3_inflow_outlet": dict(p=3, n_elems=(12, 4), box=(3.0, 0.8), geometry=A.GEOM_WALL_PROFILE,
                                       profile=A.PROFILE_GAUSS_BUMP, geom_params=(-1.5, 0.0625, 25.0, 0.0),
                                       bcs={A.LEFT: (A.BC_SUBSONIC_INFLOW, None, (1.0, 1.0, 1.0, 0.0)),
                                            A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (0.84,)),
                                            A.BOTTOM: A.BC_SLIP_WALL, A.TOP: A.BC_SLIP_WALL}),
    "wedge_bump_rusanov_p2_dirichlet": dict(p=2, n_elems=(10, 5), geometry=A.GEOM_WALL_PROFILE,
                                            profile=A.PROFILE_WEDGE_BUMP, riemann="rusanov",
                                            bcs={A.LEFT: (A.BC_DIRICHLET, (1.0, 2.0, 0.0, 4.5), None),
                                                 A.TOP: (A.BC_DIRICHLET, (1.0, 2.0, 0.0, 4.5), None),
                                                 A.RIGHT: OUT, A.BOTTOM: A.BC_SLIP_WALL}),
    "wedge_bc_hllc_p3": dict(p=3, n_elems=(8, 4), geometry=A.GEOM_WALL_PROFILE, profile=A.PROFILE_WEDGE_BC,
                             bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: A.BC_WALL, A.BOTTOM: A.BC_SLIP_WALL}),
    "delaval_hllc_p3": dict(p=3, geometry=A.GEOM_DELAVAL, bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: A.BC_WALL,
                                                                A.BOTTOM: A.BC_WALL}),
    "vortex_dirichlet_p3": dict(p=3, n_elems=(6, 6), box=(10.0, 10.0),
                                bcs={A.LEFT: VORTEX, A.RIGHT: VORTEX, A.TOP: PER, A.BOTTOM: PER}),
    "vdw_pressure_outlet_p4": dict(p=4, n_elems=(6, 4), **VDW,
                                   bcs={A.LEFT: OUT, A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (0.9,)),
                                        A.TOP: A.BC_WALL, A.BOTTOM: A.BC_WALL}),
}



CASES_1D = {
    "sod_rusanov_p3": dict(p=3, n_elems=(40, 1), riemann="rusanov", apply_filter=True),
    "hllc_p2_periodic": dict(p=2, n_elems=(33, 1), riemann="hllc", bcs={A.LEFT: PER, A.RIGHT: PER}),
    "vdw_hllc_p5_walls": dict(p=5, n_elems=(37, 1), riemann="hllc", **VDW, bcs={A.LEFT: A.BC_WALL, A.RIGHT: A.BC_WALL}),
    "dirichlet_rusanov_p4": dict(p=4, n_elems=(20, 1), riemann="rusanov",
                                 bcs={A.LEFT: (A.BC_DIRICHLET, (1.0, 0.2, 2.6), None), A.RIGHT: OUT}),
    "radial_hllc_p3": dict(p=3, n_elems=(50, 1), riemann="hllc", coord_sys=A.COORD_RADIAL,
                           bcs={A.LEFT: A.BC_WALL, A.RIGHT: OUT}),
    "p9_rusanov": dict(p=9, n_elems=(9, 1), riemann="rusanov"),
    "p1_hllc_periodic": dict(p=1, n_elems=(70, 1), riemann="hllc", bcs={A.LEFT: PER, A.RIGHT: PER}),
}


def cfg1d(name: str, **over):
    kw = dict(dim=1, box=(1.0, 1.0), bcs={A.LEFT: OUT, A.RIGHT: OUT})
    kw.update(CASES_1D[name])
    kw.update(over)
    return make_config(**kw)


# Small cases whose outputs the reference's own code (oracle/_ref) wrote into
# tests/golden/ref_<name>.npz (tests/golden/gen_ref_golden.py).  Each entry: the
# parity case it shrinks and the mesh it uses.
REF_FIXTURES_2D = {
    "cart_ideal_rusanov_p3": (4, 3),
    "cart_ideal_hllc_p1_periodic": (4, 3),
    "cart_vdw_hllc_p4_walls": (3, 3),
    "cart_vdw_rusanov_p5_perx": (3, 3),
    "cart_ideal_hllc_p6": (3, 2),
    "cart_vdw_hllc_p8_periodic": (2, 2),
    "sinewarp_hllc_p4_periodic": (3, 3),
    "bump_hllc_p3_inflow_outlet": (6, 2),
    "wedge_bump_rusanov_p2_dirichlet": (5, 3),
    "delaval_hllc_p3": (4, 3),
    "vortex_dirichlet_p3": (3, 3),
}
REF_FIXTURES_1D = ("sod_rusanov_p3", "vdw_hllc_p5_walls", "radial_hllc_p3", "dirichlet_rusanov_p4")


def ref_fixture_cfg(name: str, **over):
    """Configuration of reference fixture `name` (2D names as in REF_FIXTURES_2D, 1D
    names prefixed with '1d_')."""
    if name.startswith("1d_"):
        c = cfg1d(name[3:], **over)
        c.n_elems[0] = min(c.n_elems[0], 12)
        return c
    kw = dict(CASES_2D[name])
    kw["n_elems"] = REF_FIXTURES_2D[name]
    kw.update(over)
    return _cfg2d(**kw)
