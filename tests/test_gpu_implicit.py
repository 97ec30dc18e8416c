"""GPU: the implicit path -- coloured complex-step Jacobian blocks, the block-Jacobi
preconditioner and backward Euler with Newton-GMRES.

The oracle reference for the blocks is colouring-free: column (e, d) of the
Jacobian from the oracle's complex-step JVP with a single unit seed, restricted to
element e's rows.  Bar: TOL_JVP (the complex-step JVP tolerance).
"""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.implicit import BackwardEulerNewtonKrylov, march_to_steady
from fr_sdg_b200.workloads import bump_channel, make_config
from oracle.oracle import Oracle
from tests.helpers import TOL_JVP, cons_to_prim, random_state, rel_err

pytestmark = pytest.mark.gpu

PER = (A.BC_PERIODIC, None, None)
OUT = A.BC_OUTFLOW
BUMP_BCS = {A.LEFT: (A.BC_SUBSONIC_INFLOW, None, (1.0, 1.0, 1.0, 0.0)),
            A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (0.84,)),
            A.BOTTOM: A.BC_SLIP_WALL, A.TOP: A.BC_SLIP_WALL}

CASES = {
    # wall-profile bump, inflow / pressure outlet / slip walls, h = 1e-30 as in the bump runs
    "bump_hllc_p2": (dict(p=2, n_elems=(6, 3), box=(3.0, 0.8), riemann="hllc", geometry=A.GEOM_WALL_PROFILE,
                          profile=A.PROFILE_GAUSS_BUMP, geom_params=(-1.5, 0.0625, 25.0, 0.0), bcs=BUMP_BCS,
                          csd_eps=1e-30), 5.0),
    # odd periodic counts: the three-colour cycle colouring
    "periodic_odd_vdw_rusanov_p2": (dict(p=2, n_elems=(5, 3), riemann="rusanov", gas="vdw", vdw=(0.05, 0.02),
                                         bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}), 2.0),
    # change of variables: the state is (log rho, u, v, log e)
    "cond_sys_hllc_p1": (dict(p=1, n_elems=(4, 4), riemann="hllc", cond_sys=True,
                              bcs={A.LEFT: OUT, A.RIGHT: OUT, A.TOP: A.BC_WALL, A.BOTTOM: OUT}), 3.0),
    # curved (sine-warped) periodic mesh, even counts: checkerboard colouring
    "sinewarp_hllc_p3": (dict(p=3, n_elems=(4, 4), box=(2.0, 2.0), riemann="hllc", geometry=A.GEOM_SINE_WARP,
                              geom_params=(0.05, 0, 0, 0), bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER,
                                                                A.BOTTOM: PER}), 0.0),
}


def _state(cfg, seed):
    U = random_state(cfg, seed, amp=0.3)
    return cons_to_prim(cfg, U) if cfg.cond_sys else U


def oracle_blocks(cfg, U, t, sigma):
    """[elem][col][row] diagonal blocks from single-seed oracle JVPs."""
    o = Oracle(cfg, threads=4)
    n = cfg.poly_deg + 1
    nd = 4 * n * n
    nel = cfg.n_elems[0] * cfg.n_elems[1]
    out = np.zeros((nel, nd, nd))
    V = np.zeros_like(U)
    for e in range(nel):
        for c in range(nd):
            V[e * nd + c] = 1.0
            out[e, c] = o.jvp(t, sigma, U, V)[e * nd:(e + 1) * nd]
            V[e * nd + c] = 0.0
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_jac_blocks_match_oracle(name, cuda):
    kw, sigma = CASES[name]
    cfg = make_config(dim=2, **kw)
    U = _state(cfg, 11)
    ref = oracle_blocks(cfg, U, 0.3, sigma)
    with FRSolver(cfg) as s:
        nd = s.n_dofs // s.n_elems
        blocks = torch.full((s.n_elems * nd * nd,), float("nan"), dtype=torch.float64, device=cuda)
        s.jac_blocks(0.3, sigma, torch.from_numpy(U).to(cuda), blocks)
        got = blocks.view(s.n_elems, nd, nd).cpu().numpy()
    err = rel_err(got, ref)
    assert err <= TOL_JVP, f"{name}: rel err {err:.3e}"


def test_block_jacobi_inverts_blocks(cuda):
    kw, sigma = CASES["bump_hllc_p2"]
    cfg = make_config(dim=2, **kw)
    U = _state(cfg, 5)
    with FRSolver(cfg) as s:
        nd = s.n_dofs // s.n_elems
        Ud = torch.from_numpy(U).to(cuda)
        blocks = torch.empty(s.n_elems * nd * nd, dtype=torch.float64, device=cuda)
        s.jac_blocks(0.0, sigma, Ud, blocks)
        B = blocks.view(s.n_elems, nd, nd).transpose(1, 2)  # row-major view of each block
        x = torch.randn(s.n_dofs, dtype=torch.float64, device=cuda, generator=torch.Generator(cuda).manual_seed(3))
        r = torch.bmm(B, x.view(s.n_elems, nd, 1)).reshape(-1).contiguous()
        s.pc_setup(0.0, sigma, Ud)
        z = torch.empty_like(r)
        s.pc_apply(r, z)
        err = float((z - x).abs().max() / x.abs().max())
    assert err < 1e-4, f"block-Jacobi apply error {err:.3e} (FP32 inverses)"


def _bump_cfg(n_elems, exact):
    kw, _ = CASES["bump_hllc_p2"]
    cfg = make_config(dim=2, **{**kw, "n_elems": n_elems})
    cfg.jvp_exact_bc = exact
    return cfg


def test_exact_bc_jvp_matches_central_differences(cuda):
    """jvp_exact_bc = 1: the complex-step JVP through the inflow, outlet and slip-wall
    ghosts against central differences of the oracle residual (a test of the
    derivative, not of the reference's constant-ghost convention)."""
    cfg = _bump_cfg((6, 3), 1)
    U = random_state(cfg, 7, amp=0.05, smooth=True)
    V = np.random.default_rng(8).uniform(-1, 1, U.size) * np.abs(U)
    o = Oracle(cfg, threads=4)
    eps = 1e-6
    fd = (o.residual(0.0, U + eps * V) - o.residual(0.0, U - eps * V)) / (2 * eps)
    with FRSolver(cfg) as s:
        Ud, Vd = torch.from_numpy(U).to(cuda), torch.from_numpy(V).to(cuda)
        JV = torch.empty_like(Ud)
        s.pre_jv_eval(0.0, Ud, 0.0)
        s.matmult(Vd, JV)
        got = JV.cpu().numpy()
        # the blocks of the same Jacobian: single-seed columns of element 4
        nd = s.n_dofs // s.n_elems
        blocks = torch.empty(s.n_elems * nd * nd, dtype=torch.float64, device=cuda)
        s.jac_blocks(0.0, 0.0, Ud, blocks)
        B = blocks.view(s.n_elems, nd, nd).cpu().numpy()
        e = 4
        for c in (0, 5, nd - 1):
            seed = torch.zeros_like(Ud)
            seed[e * nd + c] = 1.0
            s.matmult(seed, JV)
            col = JV.cpu().numpy()[e * nd:(e + 1) * nd]
            assert rel_err(B[e, c], col) <= TOL_JVP
    err = rel_err(got, fd)
    assert err <= 1e-6, f"exact-BC JVP vs central differences: {err:.3e}"
    # the default convention differs exactly there: ghosts held constant
    cfg0 = _bump_cfg((6, 3), 0)
    with FRSolver(cfg0) as s0:
        JV0 = torch.empty_like(Ud)
        s0.pre_jv_eval(0.0, Ud, 0.0)
        s0.matmult(Vd, JV0)
    assert rel_err(JV0.cpu().numpy(), fd) > 1e3 * err


def test_backward_euler_newton_converges(cuda):
    """One backward-Euler step of the bump channel (inflow, outlet, slip walls, exact
    boundary derivatives) from its uniform initial state: Newton-GMRES drives ||F||
    down by 1e-8 in a few iterations, and the block-Jacobi preconditioner cuts the
    Krylov iterations."""
    wl = bump_channel(nx=12, ny=4, p=2)
    its = {}
    with FRSolver(wl.cfg) as s:
        for pc in (True, False):
            U = wl.init(cuda)
            nk = BackwardEulerNewtonKrylov(s, gmres_rtol=1e-6, newton_rtol=1e-8, max_newton=8, precondition=pc)
            st = nk.step(U, 0.0, 0.05)
            assert st.f_norms[-1] <= 1e-8 * st.f_norms[0], st.f_norms
            assert st.newton_iterations <= 5, st.f_norms
            assert s.status() == 0
            its[pc] = st.gmres_iterations
    assert its[True] < its[False], its


def test_bump_marches_to_steady(cuda):
    """Pseudo-transient continuation of the subsonic bump (24 x 8, p = 2) from the
    uniform inflow state: the steady residual drops by 1e-8."""
    wl = bump_channel(nx=24, ny=8, p=2)
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        st = march_to_steady(s, U, dt0=0.5, drop=1e-8, max_steps=40)
        assert s.status() == 0
    assert st.residual_drop <= 1e-8, st.history[-5:]


def _slot(nx, ny, per_x, per_y, e, ep):
    """Slot of element ep in element e's five-block row (0 self, 1 right, 2 top,
    3 bottom, 4 left), or None when ep is not a face neighbour."""
    i, j = e % nx, e // nx
    for s, (di, dj) in enumerate(((0, 0), (1, 0), (0, 1), (0, -1), (-1, 0))):
        ii, jj = i + di, j + dj
        if per_x:
            ii %= nx
        if per_y:
            jj %= ny
        if 0 <= ii < nx and 0 <= jj < ny and jj * nx + ii == ep:
            return s
    return None


@pytest.mark.parametrize("name,kw", [
    ("bump_hllc_p2", CASES["bump_hllc_p2"][0]),
    ("periodic_5x5_vdw_p1", dict(p=1, n_elems=(5, 5), riemann="rusanov", gas="vdw", vdw=(0.05, 0.02),
                                 bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER})),
])
def test_jac_blocks5_match_oracle(name, kw, cuda):
    cfg = make_config(dim=2, **kw)
    U = _state(cfg, 13)
    nx, ny = cfg.n_elems[0], cfg.n_elems[1]
    per_x, per_y = cfg.bc[A.LEFT].kind == A.BC_PERIODIC, cfg.bc[A.TOP].kind == A.BC_PERIODIC
    n = cfg.poly_deg + 1
    nd, nel = 4 * n * n, nx * ny
    o = Oracle(cfg, threads=4)
    ref = np.zeros((nel, 5, nd, nd))
    V = np.zeros_like(U)
    for ep in range(nel):
        for d in range(nd):
            V[ep * nd + d] = 1.0
            jv = o.jvp(0.1, 2.0, U, V)
            V[ep * nd + d] = 0.0
            for e in range(nel):
                s = _slot(nx, ny, per_x, per_y, e, ep)
                if s is not None:
                    ref[e, s, d] = jv[e * nd:(e + 1) * nd]
    with FRSolver(cfg) as sv:
        B = torch.full((nel * 5 * nd * nd,), float("nan"), dtype=torch.float64, device=cuda)
        sv.jac_blocks5(0.1, 2.0, torch.from_numpy(U).to(cuda), B)
        got = B.view(nel, 5, nd, nd).cpu().numpy()
    err = rel_err(got, ref)
    assert err <= TOL_JVP, f"{name}: rel err {err:.3e}"


def test_block_gs_sweep_matches_dense(cuda):
    """The red-black block Gauss-Seidel apply against the same sweep written densely on
    the host from the same blocks (FP32 storage: 1e-5)."""
    kw, sigma = CASES["bump_hllc_p2"]
    cfg = make_config(dim=2, **kw)
    U = _state(cfg, 5)
    nx, ny = cfg.n_elems[0], cfg.n_elems[1]
    with FRSolver(cfg) as s:
        nd = s.n_dofs // s.n_elems
        nel = s.n_elems
        Ud = torch.from_numpy(U).to(cuda)
        B5 = torch.empty(nel * 5 * nd * nd, dtype=torch.float64, device=cuda)
        s.jac_blocks5(0.0, sigma, Ud, B5)
        s.pc_setup_gs(0.0, sigma, Ud)
        r = torch.from_numpy(np.random.default_rng(6).uniform(-1, 1, s.n_dofs)).to(cuda)
        z = torch.empty_like(r)
        s.pc_apply(r, z)
        got = z.cpu().numpy().reshape(nel, nd)
    Bk = B5.view(nel, 5, nd, nd).cpu().numpy().transpose(0, 1, 3, 2)  # row-major blocks
    R = r.cpu().numpy().reshape(nel, nd)
    Dinv = [np.linalg.inv(Bk[e, 0]) for e in range(nel)]
    nb = lambda e: [(1, e + 1 if e % nx + 1 < nx else None), (2, e + nx if e // nx + 1 < ny else None),
                    (3, e - nx if e // nx > 0 else None), (4, e - 1 if e % nx > 0 else None)]
    red = [e for e in range(nel) if (e % nx + e // nx) % 2 == 0]
    black = [e for e in range(nel) if (e % nx + e // nx) % 2 == 1]
    Z = np.zeros_like(R)
    for e in red:
        Z[e] = Dinv[e] @ R[e]
    for e in black:
        Z[e] = Dinv[e] @ (R[e] - sum(Bk[e, sl] @ Z[q] for sl, q in nb(e) if q is not None))
    for e in red:
        Z[e] = Z[e] - Dinv[e] @ sum(Bk[e, sl] @ Z[q] for sl, q in nb(e) if q is not None)
    err = np.max(np.abs(got - Z)) / np.max(np.abs(Z))
    assert err < 1e-5, f"block GS apply error {err:.3e}"


def test_gs_preconditioner_beats_jacobi(cuda):
    """One backward-Euler step of the bump channel with a large time step: block
    Gauss-Seidel needs fewer Krylov iterations than block-Jacobi, same Newton result."""
    wl = bump_channel(nx=24, ny=8, p=2)
    its, fin = {}, {}
    with FRSolver(wl.cfg) as s:
        for pc in ("gs", "jacobi"):
            U = wl.init(cuda)
            nk = BackwardEulerNewtonKrylov(s, restart=60, gmres_rtol=1e-6, max_gmres=600, newton_rtol=1e-8,
                                           max_newton=8, precondition=pc)
            st = nk.step(U, 0.0, 2.0)
            assert st.f_norms[-1] <= 1e-8 * st.f_norms[0], (pc, st.f_norms)
            its[pc] = st.gmres_iterations
            fin[pc] = U.clone()
    assert its["gs"] < its["jacobi"], its
    assert float((fin["gs"] - fin["jacobi"]).abs().max()) < 1e-6


def test_coarse_operator_matches_single_probes(cuda):
    """The coarse operator from 20 coloured JVP probes equals the one probed one coarse
    unknown at a time (the bump's Jacobian, with differentiated boundary ghosts)."""
    from fr_sdg_b200.implicit import CoarseCorrection

    wl = bump_channel(nx=12, ny=4, p=2)
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        s.pre_jv_eval(0.0, U, 2.0)
        cc = CoarseCorrection(wl.cfg, 2, 2)
        got = cc.assemble(s.matmult, U)
        e, w = torch.empty_like(U), torch.empty_like(U)
        ref = torch.empty_like(got)
        for k in range(cc.nc):
            zc = torch.zeros(cc.nagg, 4, dtype=torch.float64, device=cuda)
            zc.view(-1)[k] = 1.0
            s.matmult(cc.prolong(zc, e), w)
            ref[:, k] = cc.restrict(w).reshape(-1)
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err <= 1e-12, err


def test_two_level_cuts_krylov_iterations(cuda):
    """One large backward-Euler step of the bump: the aggregate coarse level in front of
    block Gauss-Seidel needs fewer Krylov iterations for the same Newton result."""
    wl = bump_channel(nx=24, ny=8, p=2)
    its, fin = {}, {}
    with FRSolver(wl.cfg) as s:
        for name, coarse in (("gs", None), ("gs+coarse", (2, 2))):
            U = wl.init(cuda)
            nk = BackwardEulerNewtonKrylov(s, restart=60, gmres_rtol=1e-6, max_gmres=600, newton_rtol=1e-8,
                                           max_newton=8, precondition="gs", coarse=coarse)
            st = nk.step(U, 0.0, 20.0)
            assert st.f_norms[-1] <= 1e-8 * st.f_norms[0], (name, st.f_norms)
            its[name] = st.gmres_iterations
            fin[name] = U.clone()
    assert its["gs+coarse"] < its["gs"], its
    assert float((fin["gs"] - fin["gs+coarse"]).abs().max()) < 1e-6


def test_full_bump_reaches_steady_state(cuda):
    """The full bump channel (256 x 64, p = 3, 1,048,576 DOF) marched in pseudo time to
    a 1e-10 residual drop with the aggregate coarse level in front of block
    Gauss-Seidel (block Gauss-Seidel alone stalls near 2e-3 on this mesh)."""
    wl = bump_channel()
    with FRSolver(wl.cfg) as s:
        U = wl.init(cuda)
        nk = BackwardEulerNewtonKrylov(s, restart=60, max_gmres=400, max_newton=1, precondition="gs",
                                       coarse=(4, 4))
        st = march_to_steady(s, U, dt0=0.05, drop=1e-10, max_steps=40, newton=nk, max_rejections=30,
                             max_growth=3.0, reject_growth=1.5)
        assert s.status() == 0
    assert st.residual_drop <= 1e-10, st.history[-6:]


# ---- GMRES with the Arnoldi step on the device (frsdg_gmres_arnoldi) -------------------
def _dense_system(n, seed):
    g = torch.Generator().manual_seed(seed)
    Am = torch.eye(n, dtype=torch.float64) + 0.3 * torch.randn(n, n, generator=g, dtype=torch.float64) / n ** 0.5
    b = torch.randn(n, generator=g, dtype=torch.float64)
    return Am, b


@pytest.mark.parametrize("restart", [7, 30])
def test_device_gmres_matches_host_arnoldi(restart, cuda):
    """The device Arnoldi step against its host restatement on the same system: the
    same solution, and the device run takes at most two extra steps (its convergence
    check reads the residual norm two steps late)."""
    from fr_sdg_b200.implicit import gmres

    Am, b = _dense_system(2000, 5)
    xh, sh = gmres(lambda v, o: o.copy_(Am @ v), lambda r, z: z.copy_(r), b, restart=restart, rtol=1e-9,
                   max_iter=400)
    Ad, bd = Am.to(cuda), b.to(cuda)
    xd, sd = gmres(lambda v, o: torch.mv(Ad, v, out=o), lambda r, z: z.copy_(r), bd, restart=restart, rtol=1e-9,
                   max_iter=400)
    assert 0 <= sd.iterations - sh.iterations <= 2
    assert sd.residual <= 1e-9
    true_rel = float(torch.linalg.vector_norm(bd - Ad @ xd) / torch.linalg.vector_norm(bd))
    assert true_rel <= 2e-9
    assert float(torch.linalg.vector_norm(xd.cpu() - xh) / torch.linalg.vector_norm(xh)) <= 1e-8


def test_device_gmres_breakdown_and_repeatability(cuda):
    """A = 2 I: the Krylov space closes after one step (||w|| = 0); the solution is exact
    and the extra steps after the breakdown leave it alone.  Two solves of the same
    system give identical bits (fixed-order reductions)."""
    from fr_sdg_b200.implicit import gmres

    b = torch.randn(10_000, dtype=torch.float64, device=cuda)
    x, st = gmres(lambda v, o: torch.mul(v, 2.0, out=o), lambda r, z: z.copy_(r), b, restart=10, rtol=1e-12)
    assert torch.allclose(x, 0.5 * b, rtol=0, atol=1e-14)
    assert st.residual <= 1e-12
    Am, bb = _dense_system(3000, 9)
    Ad, bd = Am.to(cuda), bb.to(cuda)
    run = lambda: gmres(lambda v, o: torch.mv(Ad, v, out=o), lambda r, z: z.copy_(r), bd, restart=20, rtol=1e-10,
                        max_iter=300)[0]
    assert torch.equal(run(), run())


def test_arnoldi_step_orthogonality(cuda):
    """After m device Arnoldi steps on D = diag(1 + U(0, 1)) the basis is orthonormal to
    rounding: D v_j lies mostly along v_j (||w|| drops below 1/sqrt(2) of its value in the
    first Gram-Schmidt pass), so every step takes the second pass."""
    from fr_sdg_b200.implicit import _DeviceArnoldi

    n, m = 50_000, 12
    g = torch.Generator(device=cuda).manual_seed(3)
    d = 1.0 + torch.rand(n, generator=g, dtype=torch.float64, device=cuda)
    V = torch.zeros((m + 1, n), dtype=torch.float64, device=cuda)
    V[0] = torch.randn(n, generator=g, dtype=torch.float64, device=cuda)
    V[0] /= torch.linalg.vector_norm(V[0])
    H = torch.zeros((m + 1, m), dtype=torch.float64, device=cuda)
    cs, sn = torch.zeros(m, dtype=torch.float64, device=cuda), torch.zeros(m, dtype=torch.float64, device=cuda)
    gg = torch.zeros(m + 1, dtype=torch.float64, device=cuda)
    gg[0] = 1.0
    inv = torch.zeros(1, dtype=torch.float64, device=cuda)
    w = torch.empty(n, dtype=torch.float64, device=cuda)
    step = _DeviceArnoldi(n, cuda)
    for j in range(m):
        torch.mul(d, V[j], out=w)
        step.arnoldi(V, j, w, H, cs, sn, gg, inv)
        torch.mul(w, inv, out=V[j + 1])
    Q = V[:m]
    err = float((Q @ Q.T - torch.eye(m, dtype=torch.float64, device=cuda)).abs().max())
    assert err <= 1e-12
