"""Iterate-level pin of the oracle's restarted GMRES without JAX: one cycle
of left-preconditioned GMRES with Krylov dimension k returns, by definition,
x0 + V y with y minimising ||M (b - A (x0 + V y))|| over the Krylov space
K_k(M A, M (b - A x0)) -- the semantics of jax.scipy.sparse.linalg.gmres
(left preconditioning, ``restart`` the Krylov dimension, ``maxiter`` the
number of cycles) that the oracle restates (oracle/linalg.py).  The
minimiser is formed independently here by dense least squares; a second
cycle restarts from the first cycle's iterate.  CPU, float64."""

import pytest
import torch

from oracle.linalg import gmres


def _minres_cycle(A, M, b, x0, k):
    """x0 + V y*, V an orthonormal basis of K_k(MA, M r0), y* the dense
    least-squares minimiser of the preconditioned residual."""
    r0 = M @ (b - A @ x0)
    cols = [r0 / torch.linalg.vector_norm(r0)]
    for _ in range(k - 1):  # Arnoldi with two Gram-Schmidt passes (a well-conditioned basis)
        v = M @ (A @ cols[-1])
        for _ in range(2):
            Q = torch.stack(cols, 1)
            v = v - Q @ (Q.T @ v)
        cols.append(v / torch.linalg.vector_norm(v))
    V = torch.stack(cols, 1)
    y = torch.linalg.lstsq(M @ A @ V, r0[:, None]).solution[:, 0]
    return x0 + V @ y


def _system(n, seed):
    gen = torch.Generator().manual_seed(seed)
    A = torch.eye(n, dtype=torch.float64) * 3.0 + 0.6 * torch.randn(n, n, generator=gen, dtype=torch.float64) / n ** 0.5
    M = torch.diag(1.0 / torch.diagonal(A)) + 0.05 * torch.randn(n, n, generator=gen, dtype=torch.float64) / n ** 0.5
    b = torch.randn(n, generator=gen, dtype=torch.float64)
    x0 = 0.1 * torch.randn(n, generator=gen, dtype=torch.float64)
    return A, M, b, x0


@pytest.mark.parametrize("method", ["batched", "incremental"])
@pytest.mark.parametrize("k", [1, 3, 8])
def test_one_cycle_is_the_krylov_minimiser(method, k):
    A, M, b, x0 = _system(60, 3 + k)
    x = gmres(lambda v: A @ v, b, x0, tol=1e-30, restart=k, maxiter=1, M=lambda v: M @ v, solve_method=method)
    ref = _minres_cycle(A, M, b, x0, k)
    assert float(torch.linalg.vector_norm(x - ref) / torch.linalg.vector_norm(ref)) < 1e-10


@pytest.mark.parametrize("method", ["batched", "incremental"])
def test_second_cycle_restarts_from_the_first(method):
    A, M, b, x0 = _system(50, 11)
    k = 4
    x = gmres(lambda v: A @ v, b, x0, tol=1e-30, restart=k, maxiter=2, M=lambda v: M @ v, solve_method=method)
    ref = _minres_cycle(A, M, b, _minres_cycle(A, M, b, x0, k), k)
    assert float(torch.linalg.vector_norm(x - ref) / torch.linalg.vector_norm(ref)) < 1e-10


def test_cycle_count_and_early_stop():
    """``maxiter`` counts restart cycles and the outer test is on the
    preconditioned residual against max(tol ||b||, atol)."""
    A, M, b, x0 = _system(40, 5)
    st = {}
    gmres(lambda v: A @ v, b, x0, tol=1e-8, restart=5, maxiter=50, M=lambda v: M @ v, stats=st)
    assert 1 < st["cycles"] < 50 and st["residual_norm"] <= st["atol"]
    assert abs(st["atol"] - 1e-8 * float(torch.linalg.vector_norm(b))) < 1e-20
    st2 = {}
    gmres(lambda v: A @ v, b, x0, tol=1e-8, restart=5, maxiter=2, M=lambda v: M @ v, stats=st2)
    assert st2["cycles"] == 2 and st2["arnoldi_steps"] == 10
