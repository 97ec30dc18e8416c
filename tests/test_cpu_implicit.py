"""CPU: the host side of the implicit path (right-preconditioned GMRES)."""
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
