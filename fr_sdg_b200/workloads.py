"""Configurations and synthetic initial states of the five benchmark workloads.

Each builder returns a `Workload` with the handle configuration (a
`frsdg_config`), the time-integration settings and a function that fills the
initial state in the DMDA natural layout on a torch device.  The initial
states restate the reference's problem factory (include/factory.hpp): the Sod
tube (175-229), the isentropic vortex (311-395) and the circular explosion
(400-465); the bump channel and the large blast are the synthetic inputs named
by the workload descriptions.  Initial conditions are evaluated at the physical
node coordinates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import torch

from . import _abi as A
from .refelem import reference_element


def make_config(dim: int = 2, p: int = 3, n_elems=(10, 10), box=(1.0, 1.0), radau_corr: float = 0.0,
                gas: str = "ideal", gamma: float = 1.4, vdw=(161.94, 0.001265), riemann: str = "rusanov",
                geometry: int = A.GEOM_CARTESIAN, profile: int = A.PROFILE_FLAT, geom_params=(0.0, 0.0, 0.0, 0.0),
                bcs=None, apply_filter: bool = False, cut_off: int = 2, strength: int = 32, alpha: float = 36.0,
                apply_weno: bool = False, weno_gamma: float = 0.998, theta: float = 1.0, threshold: float = 0.8,
                cond_sys: bool = False, csd_eps: float = 1e-7, coord_sys: int = A.COORD_CARTESIAN,
                pp_limit: bool = False, pp_eps: float = 1e-13,
                defaults: Callable[[A.frsdg_config], None] | None = None) -> A.frsdg_config:
    """Build a configuration; `bcs` maps a face (A.LEFT..A.BOTTOM) to a kind or
    to (kind, state, params).  The remaining fields take the library's defaults
    (frsdg_config_default), or those `defaults(cfg)` writes."""
    c = A.frsdg_config()
    if defaults is None:
        A.check(A.lib().frsdg_config_default(c), "frsdg_config_default")
    else:
        defaults(c)
    c.dim, c.poly_deg = dim, p
    c.n_elems[0] = n_elems[0]
    c.n_elems[1] = n_elems[1] if dim == 2 else 1
    c.box_length[0] = box[0]
    c.box_length[1] = box[1] if dim == 2 else 1.0
    c.radau_corr = radau_corr
    c.gas_law = {"ideal": A.GAS_IDEAL, "vdw": A.GAS_VDW}[gas]
    c.gamma = gamma
    c.vdw_a, c.vdw_b = vdw
    c.riemann = {"rusanov": A.RUSANOV, "hllc": A.HLLC}[riemann]
    c.coord_sys = coord_sys
    c.geometry, c.geom_profile = geometry, profile
    for i, v in enumerate(geom_params):
        c.geom_params[i] = v
    for face, spec in (bcs or {}).items():
        if isinstance(spec, int):
            c.bc[face].kind = spec
        else:
            kind, state, params = spec
            c.bc[face].kind = kind
            for i, v in enumerate(state or ()):
                c.bc[face].state[i] = v
            for i, v in enumerate(params or ()):
                c.bc[face].params[i] = v
    c.apply_filter, c.filt_cut_off, c.filt_strength, c.filt_alpha = int(apply_filter), cut_off, strength, alpha
    c.apply_weno, c.weno_gamma, c.shock_theta, c.shock_threshold = int(apply_weno), weno_gamma, theta, threshold
    c.cond_sys, c.csd_eps = int(cond_sys), csd_eps
    c.pp_limit, c.pp_eps = int(pp_limit), pp_eps
    return c


# ---------------------------------------------------------------- geometry on the host
def node_coords(cfg: A.frsdg_config, device="cpu", rows: tuple[int, int] | None = None,
                gll_nodes=None) -> tuple[torch.Tensor, torch.Tensor]:
    """Physical (x, y) of every node, shaped (Ny, Nx, n, n) [j, i, l, k] (2D) or
    (Nx, n) (1D).  Same analytic maps as the library's geometry policies.
    rows = (row_base, count): only `count` element rows from global row `row_base`
    (rows outside [0, Ny) wrap around, as the ghost rows of a periodic partition).
    gll_nodes: the p + 1 GLL nodes to use (default: the library's reference element)."""
    p = cfg.poly_deg
    nodes = reference_element(p)[0] if gll_nodes is None else gll_nodes
    x_ref = torch.tensor(nodes, dtype=torch.float64, device=device)
    if cfg.dim == 1:
        N = cfg.n_elems[0]
        h = cfg.box_length[0] / N
        e = torch.arange(N, dtype=torch.float64, device=device)[:, None]
        return h * (e + 0.5 * (1.0 + x_ref[None, :])), None
    Nx, Ny = cfg.n_elems[0], cfg.n_elems[1]
    i = torch.arange(Nx, dtype=torch.float64, device=device)
    if rows is None:
        j = torch.arange(Ny, dtype=torch.float64, device=device)
    else:
        j = torch.remainder(torch.arange(rows[0], rows[0] + rows[1], device=device), Ny).to(torch.float64)
    csi = (1.0 / Nx) * (i[None, :, None, None] + 0.5 * (1.0 + x_ref[None, None, None, :]))
    eta = (1.0 / Ny) * (j[:, None, None, None] + 0.5 * (1.0 + x_ref[None, None, :, None]))
    csi, eta = torch.broadcast_tensors(csi, eta)
    Lx, Ly = cfg.box_length[0], cfg.box_length[1]
    g = cfg.geometry
    if g == A.GEOM_SINE_WARP:
        d = cfg.geom_params[0] * torch.sin(2 * math.pi * csi) * torch.sin(2 * math.pi * eta)
        return Lx * csi + d, Ly * eta + d
    if g == A.GEOM_DELAVAL:
        return Lx * csi, -0.5 * (1.0 - eta) + 0.5 * eta
    if g == A.GEOM_WALL_PROFILE:
        x = cfg.geom_params[0] + Lx * csi
        if cfg.geom_profile == A.PROFILE_GAUSS_BUMP:
            h = cfg.geom_params[1] * torch.exp(-cfg.geom_params[2] * x * x)
        elif cfg.geom_profile == A.PROFILE_FLAT:
            h = torch.zeros_like(x)
        else:
            raise NotImplementedError("node_coords: wedge profiles are only used through the library")
        return x, h * (1.0 - eta) + Ly * eta
    return Lx * csi, Ly * eta


def rhoE(gas: str, gamma: float, a: float, b: float, rho, vel2, p):
    """get_rhoE of the gas laws (gas_models.hpp:81-86, 144-157) with |v|^2 given."""
    if gas == "ideal":
        return p / (gamma - 1.0) + 0.5 * rho * vel2
    a_rho_sq = a * rho * rho
    return ((p + a_rho_sq) * (1.0 - b * rho)) / (gamma - 1.0) - a_rho_sq + 0.5 * rho * vel2


def pack2d(rho, ru, rv, E) -> torch.Tensor:
    """(Ny, Nx, n, n) fields -> DMDA natural order vector (j, i, l, k, eq)."""
    return torch.stack([rho, ru, rv, E], dim=-1).reshape(-1).contiguous()


def pack1d(rho, ru, E) -> torch.Tensor:
    """(N, n) fields -> 1D element-SoA vector (e, eq, node)."""
    return torch.stack([rho, ru, E], dim=1).reshape(-1).contiguous()


# ---------------------------------------------------------------- exact solutions
def exact_vortex(t: float, x, y, u0=1.0, v0=1.0, beta=5.0, r_v=1.0, l=10.0):
    """factory.hpp:311-352 (gamma fixed at 1.4 there)."""
    gamma, pi = 1.4, math.pi
    xc = l / 2.0 + u0 * t
    yc = l / 2.0 + v0 * t
    xc = xc - l * math.floor(xc / l)
    yc = yc - l * math.floor(yc / l)
    dx, dy = x - xc, y - yc
    r2 = dx * dx + dy * dy
    f = 1.0 - r2 / (r_v * r_v)
    ef = torch.exp(f)
    rho = (1.0 - (beta * beta * (gamma - 1.0) * (ef * ef)) / (16.0 * gamma * pi * pi)) ** (1.0 / (gamma - 1.0))
    u = u0 - (beta * ef * dy) / (2.0 * pi * r_v)
    v = v0 + (beta * ef * dx) / (2.0 * pi * r_v)
    p = rho ** gamma
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return rho, rho * u, rho * v, E


# ---------------------------------------------------------------- workloads
@dataclass
class Workload:
    name: str
    cfg: A.frsdg_config
    integrator: str            # "ssprk3" | "rk4" | "beuler"
    cfl: float
    t_end: float | None
    n_steps: int | None
    init: Callable[[str], torch.Tensor]
    notes: dict = field(default_factory=dict)
    cfl_rule: str = "h"        # fr_sdg_b200.integrate.cfl_time_step

    @property
    def n_nodes(self) -> int:
        n = self.cfg.poly_deg + 1
        if self.cfg.dim == 1:
            return self.cfg.n_elems[0] * n
        return self.cfg.n_elems[0] * self.cfg.n_elems[1] * n * n

    @property
    def n_dofs(self) -> int:
        return self.n_nodes * (self.cfg.dim + 2)

    def time_step(self, U0: torch.Tensor) -> float:
        """The workload's time step on the state U0 (its CFL number and rule)."""
        from .integrate import cfl_time_step

        return cfl_time_step(self.cfg, U0, self.cfl, self.cfl_rule)


# Stabilisation of the shock workloads.  Their initial jumps sit inside elements (the
# reference's factory puts the interface node on one state, factory.hpp:199), and the
# reference's stabilisation keeps neither density nor pressure positive there: run
# through fr_sdg's own code (oracle/_ref), the spectral filter alone makes the density
# negative at the first post-step (removing the top Legendre mode of a step
# overshoots), and WENO with the shock sensor loses positivity within 1-20 steps at
# p >= 4 for every CFL number down to 0.0125 and every sensor setting tried.  The
# shock workloads therefore keep the configured stabilisation and add the
# positivity-preserving limiter (Zhang and Shu 2010; cfg.pp_limit) on every stage and
# after the post-step, with the time step dt = CFL h / ((2p + 1) c_max): the (2p + 1)
# scaling of the reference tools' own explicit CFL ceilings (tools/c-vcjh_claude.py:
# 410-430, tools/cfl_ceiling_plots.py:110-130), which keeps CFL 0.1 below both the
# linear stability limit of p >= 4 in 2D and the limiter's positivity bound
# 1 / (2 p (p + 1)).
FILTER_STAB = dict(apply_filter=True, pp_limit=True)
# "spectral filter with a shock sensor active": filter and WENO + sensor both on; the
# reference then keeps the filter's result in troubled elements (filter.hpp:733-742)
FILTER_SENSOR_STAB = dict(apply_filter=True, apply_weno=True, weno_gamma=0.998, threshold=0.8, theta=1.0,
                          pp_limit=True)
# the reference tools' own shock-run settings (tools/check_radial.py:221-236): WENO with
# the shock sensor, filter off
SHOCK_STAB = dict(apply_filter=False, apply_weno=True, weno_gamma=0.998, threshold=0.8, theta=1.0)


def sod1d(n_elems: int = 200, p: int = 3) -> Workload:
    """1D Sod tube: [0,1], Rusanov, DG (c=0), SSP-RK3 to t_end 0.2, spectral filter on,
    CFL 0.1 (dt = CFL h / ((2p+1) c_max)) with the positivity limiter."""
    cfg = make_config(dim=1, p=p, n_elems=(n_elems, 1), box=(1.0, 1.0), riemann="rusanov",
                      bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW}, **FILTER_STAB)

    def init(device="cpu"):
        x, _ = node_coords(cfg, device)
        left = x < 0.5
        rho = torch.where(left, 1.0, 0.125).to(torch.float64)
        p_ = torch.where(left, 1.0, 0.1).to(torch.float64)
        zero = torch.zeros_like(rho)
        return pack1d(rho, zero, rhoE("ideal", 1.4, 0, 0, rho, zero, p_))

    return Workload(f"sod1d_n{n_elems}_p{p}", cfg, "ssprk3", 0.1, 0.2, None, init, cfl_rule="dg")


def vortex_curved(n_elems: int = 64, p: int = 4, amplitude: float = 0.1) -> Workload:
    """Isentropic vortex on the sine-warped periodic [0,10]^2 mesh, HLLC, RK4 to t=10."""
    per = (A.BC_PERIODIC, None, None)
    cfg = make_config(dim=2, p=p, n_elems=(n_elems, n_elems), box=(10.0, 10.0), riemann="hllc",
                      geometry=A.GEOM_SINE_WARP, geom_params=(amplitude, 0, 0, 0),
                      bcs={A.LEFT: per, A.RIGHT: per, A.TOP: per, A.BOTTOM: per})

    def init(device="cpu"):
        x, y = node_coords(cfg, device)
        return pack2d(*exact_vortex(0.0, x, y))

    # CFL 0.05: RK4 with p = 4 on the warped mesh diverges at 0.1 (checked with the oracle)
    return Workload(f"vortex_sinewarp_{n_elems}x{n_elems}_p{p}", cfg, "rk4", 0.05, 10.0, None, init)


def bump_channel(nx: int = 256, ny: int = 64, p: int = 3, mach: float = 0.5) -> Workload:
    """Smooth-bump channel [-1.5,1.5]x[0,0.8], wall y = 0.0625 exp(-25 x^2), HLLC,
    subsonic total-pressure inflow (p0 = T0 = 1, R = 1), pressure outlet, slip walls."""
    g = 1.4
    p0, T0, Rg = 1.0, 1.0, 1.0
    fac = 1.0 + 0.5 * (g - 1.0) * mach * mach
    p_out = p0 * fac ** (-g / (g - 1.0))
    cfg = make_config(dim=2, p=p, n_elems=(nx, ny), box=(3.0, 0.8), riemann="hllc",
                      geometry=A.GEOM_WALL_PROFILE, profile=A.PROFILE_GAUSS_BUMP,
                      geom_params=(-1.5, 0.0625, 25.0, 0.0),
                      bcs={A.LEFT: (A.BC_SUBSONIC_INFLOW, None, (p0, T0, Rg, 0.0)),
                           A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (p_out,)),
                           A.BOTTOM: A.BC_SLIP_WALL, A.TOP: A.BC_SLIP_WALL},
                      csd_eps=1e-30)
    # Newton needs the boundary ghosts differentiated: with them held constant (the
    # reference's treatment of user-lambda boundaries) the Jacobian misses the inflow,
    # outlet and slip-wall couplings and Newton stalls
    cfg.jvp_exact_bc = 1

    def init(device="cpu"):
        x, _ = node_coords(cfg, device)
        T = T0 / fac
        rho0 = p_out / (Rg * T)
        u0 = mach * math.sqrt(g * p_out / rho0)
        rho = torch.full_like(x, rho0)
        ru = rho * u0
        rv = torch.zeros_like(x)
        E = rhoE("ideal", g, 0, 0, rho, torch.full_like(x, u0 * u0), torch.full_like(x, p_out))
        return pack2d(rho, ru, rv, E)

    return Workload(f"bump_{nx}x{ny}_p{p}", cfg, "beuler", None, None, None, init,
                    notes={"p_out": p_out})


def blast_large(n_elems: int = 1024, p: int = 5, ny: int | None = None, defaults=None,
                gll_nodes=None) -> Workload:
    """2D radial blast on [0,1]^2, HLLC, Van der Waals (a=0.05, b=0.02, gamma=1.4),
    SSP-RK3, 200 steps, spectral filter with the shock sensor active and the positivity
    limiter, CFL 0.1 (dt = CFL h / ((2p+1) c_max)).  ny > n_elems stacks
    more rows of the same element size above it (box [0,1] x [0, ny/n_elems]): the
    weak-scaling mesh of a row-block partition.  `defaults` and `gll_nodes` replace
    the library's configuration defaults and reference element (make_config,
    node_coords), so that the same input can be built without the library."""
    a, b, g = 0.05, 0.02, 1.4
    ny = ny or n_elems
    cfg = make_config(dim=2, p=p, n_elems=(n_elems, ny), box=(1.0, ny / n_elems), riemann="hllc",
                      gas="vdw", gamma=g, vdw=(a, b),
                      bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_OUTFLOW,
                           A.BOTTOM: A.BC_OUTFLOW},
                      defaults=defaults, **FILTER_SENSOR_STAB)

    def init(device="cpu", rows=None):
        x, y = node_coords(cfg, device, rows, gll_nodes)
        r = torch.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2)
        inside = r < 0.4
        rho = torch.where(inside, 1.0, 0.125).to(torch.float64)
        pr = torch.where(inside, 1.0, 0.1).to(torch.float64)
        zero = torch.zeros_like(rho)
        return pack2d(rho, zero, zero, rhoE("vdw", g, a, b, rho, zero, pr))

    return Workload(f"blast_vdw_{n_elems}x{ny}_p{p}", cfg, "ssprk3", 0.1, None, 200, init, cfl_rule="dg")


def circular_explosion(n_elems: int, p: int, gas: str, gamma: float, vdw, r0: float, p_out: float,
                       filt_cut_off: int = 2) -> Workload:
    """One instance of the batched uneven workload: ProblemFactory2D<CircularExplosion>
    (factory.hpp:400-465) on [-1,1]^2 with Rusanov and outflow boundaries, spectral
    filter on with the positivity limiter, SSP-RK3 to t_end 0.25 at CFL 0.1
    (dt = CFL h / ((2p+1) c_max)).  The limiter's floor is 1e-6, four orders below the
    smallest physical pressure (0.05): with the default 1e-13 the nodes it lifts carry
    internal energies ~1e-11 of their kinetic energy, below what the FP32 arithmetic of
    the mixed form resolves."""
    cfg = make_config(dim=2, p=p, n_elems=(n_elems, n_elems), box=(2.0, 2.0), riemann="rusanov",
                      gas=gas, gamma=gamma, vdw=vdw,
                      bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_OUTFLOW,
                           A.BOTTOM: A.BC_OUTFLOW},
                      cut_off=filt_cut_off, pp_eps=1e-6, **FILTER_STAB)

    def init(device="cpu"):
        x, y = node_coords(cfg, device)
        r = torch.sqrt((x - 1.0) ** 2 + (y - 1.0) ** 2)
        inside = r < r0
        rho = torch.where(inside, 1.0, 0.125).to(torch.float64)
        pr = torch.where(inside, torch.tensor(1.0, dtype=torch.float64), torch.tensor(p_out, dtype=torch.float64))
        zero = torch.zeros_like(rho)
        return pack2d(rho, zero, zero, rhoE(gas, gamma, vdw[0], vdw[1], rho, zero, pr))

    return Workload(f"explosion_{n_elems}_p{p}_{gas}", cfg, "ssprk3", 0.1, 0.25, None, init, cfl_rule="dg")
