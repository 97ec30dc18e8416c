"""CPU: the host side of the implicit path (right-preconditioned GMRES)."""
import numpy as np
import pytest
import torch

from fr_sdg_b200.implicit import gmres


def _system(n=60, seed=0):
    g = torch.Generator().manual_seed(seed)
    A = torch.eye(n, dtype=torch.float64) * 4 + 0.3 * torch.randn(n, n, dtype=torch.float64, generator=g)
    b = torch.randn(n, dtype=torch.float64, generator=g)
    return A, b


def test_gmres_unpreconditioned_with_restarts():
    A, b = _system()
    x, st = gmres(lambda v, o: o.copy_(A @ v), lambda r, z: z.copy_(r), b, restart=10, rtol=1e-12, max_iter=300)
    assert float(torch.linalg.vector_norm(A @ x - b) / torch.linalg.vector_norm(b)) < 1e-10
    assert st.residual <= 1e-12


def test_gmres_right_preconditioned_exact_preconditioner_one_step():
    A, b = _system(40, 1)
    Ainv = torch.linalg.inv(A)
    x, st = gmres(lambda v, o: o.copy_(A @ v), lambda r, z: z.copy_(Ainv @ r), b, restart=10, rtol=1e-10)
    assert st.iterations == 1
    assert float(torch.linalg.vector_norm(A @ x - b) / torch.linalg.vector_norm(b)) < 1e-10


def test_gmres_zero_rhs():
    A, _ = _system(8)
    x, st = gmres(lambda v, o: o.copy_(A @ v), lambda r, z: z.copy_(r), torch.zeros(8, dtype=torch.float64))
    assert st.iterations == 0 and float(x.abs().max()) == 0.0


def test_gmres_residual_estimate_matches_true_residual():
    A, b = _system(50, 2)
    x, st = gmres(lambda v, o: o.copy_(A @ v), lambda r, z: z.copy_(r), b, restart=7, rtol=1e-4, max_iter=300)
    true = float(torch.linalg.vector_norm(A @ x - b) / torch.linalg.vector_norm(b))
    assert true <= 1e-4 * 1.01
    assert abs(true - st.residual) <= 1e-6


def _face_coupled_operator(nx, ny, nd, seed):
    """A random operator coupling each element to itself and its face neighbours,
    the sparsity of the residual's Jacobian on a non-periodic mesh."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nd
    J = np.zeros((n, n))
    for j in range(ny):
        for i in range(nx):
            e = j * nx + i
            for di, dj in ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < nx and 0 <= jj < ny:
                    q = jj * nx + ii
                    J[e * nd:(e + 1) * nd, q * nd:(q + 1) * nd] = rng.standard_normal((nd, nd))
    return J


@pytest.mark.parametrize("ax,ay", [(2, 2), (3, 2), (1, 1), (7, 5)])
def test_coarse_operator_by_coloured_probing(ax, ay):
    """CoarseCorrection.assemble (20 probes, aggregates coloured (I + 2J) mod 5) equals
    P^T J P formed densely, on a 7 x 5 mesh with uneven aggregates."""
    from fr_sdg_b200.implicit import CoarseCorrection
    from fr_sdg_b200.workloads import make_config

    cfg = make_config(dim=2, p=1, n_elems=(7, 5))
    nx, ny, nn = 7, 5, 4
    nd = 4 * nn
    J = torch.from_numpy(_face_coupled_operator(nx, ny, nd, seed=ax * 10 + ay))
    cc = CoarseCorrection(cfg, ax, ay)
    # explicit P: column (K, v) = indicator of variable v on every node of aggregate K
    P = torch.zeros(nx * ny * nd, cc.nc, dtype=torch.float64)
    for k in range(cc.nc):
        zc = torch.zeros(cc.nagg, 4, dtype=torch.float64)
        zc.view(-1)[k] = 1.0
        P[:, k] = cc.prolong(zc, torch.empty(nx * ny * nd, dtype=torch.float64))
    ref = P.T @ J @ P
    probes = []

    def matvec(v, out):
        probes.append(1)
        out.copy_(J @ v)

    got = cc.assemble(matvec, torch.zeros(nx * ny * nd, dtype=torch.float64))
    assert len(probes) == 20
    assert torch.allclose(got, ref, rtol=0, atol=1e-12 * float(ref.abs().max()))
    # restriction is the transpose of the prolongation
    r = torch.from_numpy(np.random.default_rng(3).standard_normal(nx * ny * nd))
    assert torch.allclose(cc.restrict(r).reshape(-1), P.T @ r, atol=1e-12)


def test_coarse_colouring_is_distance_two():
    """Every aggregate's closed five-aggregate neighbourhood has five distinct colours,
    and neighbour_of_colour finds the one of each colour."""
    from fr_sdg_b200.implicit import CoarseCorrection
    from fr_sdg_b200.workloads import make_config

    cc = CoarseCorrection(make_config(dim=2, p=1, n_elems=(23, 11)), 2, 2)
    cc._maps(torch.device("cpu"))
    gx, gy = cc.gx, cc.gy
    col = cc.colour.view(gy, gx)
    for c in range(5):
        nb = cc.neighbour_of_colour(c, torch.device("cpu"))
        for k in range(cc.nagg):
            I, Jj = k % gx, k // gx
            hood = [(I + di, Jj + dj) for di, dj in ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1))
                    if 0 <= I + di < gx and 0 <= Jj + dj < gy]
            cols = [int(col[b, a]) for a, b in hood]
            assert len(set(cols)) == len(cols)
            match = [b * gx + a for a, b in hood if int(col[b, a]) == c]
            assert int(nb[k]) == (match[0] if match else -1)


class _PseudoTimeModel:
    """Stand-ins for march_to_steady: a 'solver' whose residual norm is the first entry
    of U, and a 'Newton step' that multiplies it by 1 / (1 + dt) -- or blows it up when
    dt exceeds blow_dt (a step the march must reject)."""

    def __init__(self, blow_dt: float):
        self.blow_dt = blow_dt
        self.dts = []

    # solver side
    def residual_kernel(self, t, U, R):
        R.zero_()
        R[0] = U[0]

    def status(self):
        return 0

    # Newton side
    def step(self, U, t, dt):
        from fr_sdg_b200.implicit import NewtonStats

        self.dts.append(dt)
        U[0] = U[0] * (1e6 if dt > self.blow_dt else 1.0 / (1.0 + dt))
        return NewtonStats(1, 3)


def test_march_rejects_growth_and_caps_the_time_step():
    from fr_sdg_b200.implicit import march_to_steady

    m = _PseudoTimeModel(blow_dt=50.0)
    U = torch.ones(4, dtype=torch.float64)
    st = march_to_steady(m, U, dt0=0.5, drop=1e-10, max_steps=200, newton=m, max_growth=3.0, reject_growth=1.5)
    assert st.residual_drop <= 1e-10
    # every attempt above blow_dt grew the residual 1e6-fold and was rejected (dt / 4)
    assert st.rejected == sum(1 for dt in m.dts if dt > 50.0) and st.rejected > 0
    for a, b in zip(m.dts, m.dts[1:]):
        assert b <= 3.0 * a + 1e-12 or b == a / 4  # growth capped, or a rejection's quarter step
    assert st.gmres_iterations == 3 * len(m.dts)  # rejected attempts' Krylov work counts too


def test_march_without_rejection_rule_accepts_growth():
    from fr_sdg_b200.implicit import march_to_steady

    m = _PseudoTimeModel(blow_dt=1e9)
    U = torch.ones(4, dtype=torch.float64)
    st = march_to_steady(m, U, dt0=0.5, drop=1e-8, max_steps=100, newton=m)
    assert st.rejected == 0 and st.residual_drop <= 1e-8
    # switched evolution relaxation: dt_k = dt0 / drop_k
    assert all(abs(b - min(0.5 / d, 1e6)) < 1e-9 * b for b, d in zip(m.dts[1:], st.history[1:]))
