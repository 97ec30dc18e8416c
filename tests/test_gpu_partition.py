"""GPU: the row window of domain decomposition.  Ranks are emulated one after the
other on one GPU: each row block gets its ghost rows cut from the global state (what
the NCCL exchange delivers), and its owned rows must equal the whole-mesh results bit
for bit -- residual, RK stage, JVP and post-step."""
import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200 import _abi as A
from fr_sdg_b200.partition import row_blocks, scatter_rows
from fr_sdg_b200.workloads import make_config
from tests.helpers import random_state

pytestmark = pytest.mark.gpu

PER = (A.BC_PERIODIC, None, None)
CASES = {
    "sinewarp_periodic_hllc_p4": dict(p=4, n_elems=(6, 7), box=(10.0, 10.0), riemann="hllc",
                                      geometry=A.GEOM_SINE_WARP, geom_params=(0.1, 0, 0, 0),
                                      bcs={A.LEFT: PER, A.RIGHT: PER, A.TOP: PER, A.BOTTOM: PER}),
    "bump_inflow_outlet_p3": dict(p=3, n_elems=(12, 7), box=(3.0, 0.8), riemann="hllc",
                                  geometry=A.GEOM_WALL_PROFILE, profile=A.PROFILE_GAUSS_BUMP,
                                  geom_params=(-1.5, 0.0625, 25.0, 0.0),
                                  bcs={A.LEFT: (A.BC_SUBSONIC_INFLOW, None, (1.0, 1.0, 1.0, 0.0)),
                                       A.RIGHT: (A.BC_PRESSURE_OUTLET, None, (0.84,)),
                                       A.BOTTOM: A.BC_SLIP_WALL, A.TOP: A.BC_SLIP_WALL}),
    "vdw_walls_weno_p5": dict(p=5, n_elems=(5, 9), riemann="hllc", gas="vdw", vdw=(0.05, 0.02),
                              apply_weno=True, threshold=0.0,
                              bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW, A.TOP: A.BC_WALL,
                                   A.BOTTOM: A.BC_WALL}),
}


@pytest.mark.parametrize("ranks", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_row_blocks_reproduce_whole_mesh(name, ranks, cuda):
    cfg = make_config(dim=2, **CASES[name])
    nx, ny = cfg.n_elems[0], cfg.n_elems[1]
    U = torch.from_numpy(random_state(cfg, 9, amp=0.2)).to(cuda)
    V = torch.from_numpy(np.random.default_rng(10).uniform(-1, 1, U.numel())).to(cuda)
    periodic = cfg.bc[A.TOP].kind == A.BC_PERIODIC
    with FRSolver(cfg) as g:
        nd = g.n_dofs // (nx * ny)
        R, S, JV = torch.empty_like(U), torch.empty_like(U), torch.empty_like(U)
        g.rhs_func(0.1, U, R)
        g.rk_stage(0.1, U, S, gamma=0.01, a=U, alpha=1.0)
        g.pre_jv_eval(0.1, U, 2.0)
        g.matmult(V, JV)
        P = U.clone()
        g.apply_stabilization(P)
        with FRSolver(cfg) as s:
            for blk in row_blocks(ny, ranks, periodic):
                s.set_row_window(*blk.window())
                Ul, Vl = scatter_rows(U, blk, nx, nd), scatter_rows(V, blk, nx, nd)
                own = slice(blk.row_begin * nx * nd, blk.row_end * nx * nd)
                gown = slice(blk.g_begin * nx * nd, blk.g_end * nx * nd)
                Rl, Sl, Jl = torch.empty_like(Ul), torch.empty_like(Ul), torch.empty_like(Ul)
                s.rhs_func(0.1, Ul, Rl)
                s.rk_stage(0.1, Ul, Sl, gamma=0.01, a=Ul, alpha=1.0)
                s.pre_jv_eval(0.1, Ul, 2.0)
                s.matmult(Vl, Jl)
                Pl = Ul.clone()
                s.apply_stabilization(Pl)
                assert torch.equal(Rl[own], R[gown]), f"rank {blk.rank}: residual"
                assert torch.equal(Sl[own], S[gown]), f"rank {blk.rank}: RK stage"
                assert torch.equal(Jl[own], JV[gown]), f"rank {blk.rank}: JVP"
                assert torch.equal(Pl[own], P[gown]), f"rank {blk.rank}: post-step"
            s.set_row_window(0, 0, 0, 0)
            assert s.n_dofs == g.n_dofs


def test_row_window_rejects_bad_windows(cuda):
    cfg = make_config(dim=2, p=2, n_elems=(4, 6), bcs={A.LEFT: A.BC_OUTFLOW, A.RIGHT: A.BC_OUTFLOW,
                                                        A.TOP: A.BC_WALL, A.BOTTOM: A.BC_WALL})
    with FRSolver(cfg) as s:
        for w in [(0, 4, 1, 5), (2, 3, 0, 3), (0, 7, 0, 7), (3, 4, 1, 4), (-1, 4, 1, 4)]:
            with pytest.raises(A.FrsdgError):
                s.set_row_window(*w)
        s.set_row_window(0, 4, 0, 3)    # rank 0 of 2: ghost above only
        s.set_row_window(2, 4, 1, 4)    # last rank: ghost below only


def test_partitioned_time_stepping_matches_whole_mesh(cuda):
    """SSP-RK3 with the WENO post-step on three row blocks, each advanced by its own
    Integrator whose stage hook refreshes the ghost rows (ranks emulated by threads in
    lockstep, the exchange a device copy between their arrays), against the whole-mesh
    run: identical after 8 steps."""
    import threading

    from fr_sdg_b200.integrate import Integrator

    cfg = make_config(dim=2, **CASES["vdw_walls_weno_p5"])
    nx, ny = cfg.n_elems[0], cfg.n_elems[1]
    U0 = torch.from_numpy(random_state(cfg, 4, amp=0.05, smooth=True)).to(cuda)
    dt, steps, ranks = 2e-4, 8, 3
    with FRSolver(cfg) as g:
        nd = g.n_dofs // (nx * ny)
        Ug = U0.clone()
        Integrator(g, "ssprk3").run(Ug, dt, n_steps=steps)
    row_len = nx * nd
    blks = row_blocks(ny, ranks, periodic_y=False)
    shared, bar = {}, threading.Barrier(ranks)

    def hook_for(blk):
        def hook(V):
            torch.cuda.synchronize()
            shared[blk.rank] = V
            bar.wait()
            W = V.view(blk.rows, row_len)
            if blk.ghost_below:
                nb = blks[blk.down]
                W[0] = shared[nb.rank].view(nb.rows, row_len)[nb.row_end - 1]
            if blk.ghost_above:
                nb = blks[blk.up]
                W[blk.rows - 1] = shared[nb.rank].view(nb.rows, row_len)[nb.row_begin]
            torch.cuda.synchronize()
            bar.wait()
        return hook

    solvers = [FRSolver(cfg) for _ in blks]
    locals_, errors = [], []
    try:
        for s, blk in zip(solvers, blks):
            s.set_row_window(*blk.window())
            locals_.append(scatter_rows(U0, blk, nx, nd))

        def work(k):
            try:
                Integrator(solvers[k], "ssprk3", before_stage=hook_for(blks[k])).run(locals_[k], dt, n_steps=steps)
            except Exception as exc:  # reported below; the barrier is aborted so the others stop
                errors.append(exc)
                bar.abort()

        th = [threading.Thread(target=work, args=(k,)) for k in range(ranks)]
        for t in th:
            t.start()
        for t in th:
            t.join(timeout=300)
        assert not errors, errors
        for blk, L in zip(blks, locals_):
            own = L.view(blk.rows, row_len)[blk.row_begin:blk.row_end].reshape(-1)
            assert torch.equal(own, Ug.view(ny, row_len)[blk.g_begin:blk.g_end].reshape(-1)), blk.rank
    finally:
        for s in solvers:
            s.close()
