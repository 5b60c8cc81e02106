"""Oracle restatement of the third-party linear algebra on the SISL path.

* ``gmres``: ``jax.scipy.sparse.linalg.gmres`` (jax/jaxlib >= 0.10.0, no lock
  file in the reference; called at ``suetes/regional3d/steppers.py:466`` and
  ``:476``).  Restated from JAX's published algorithm: ``restart`` is the
  Krylov dimension and ``maxiter`` the number of restart cycles; the outer
  loop runs while ``k < maxiter`` and ``||M(b - A x)|| > atol`` with
  ``atol = max(tol * ||b||, atol)``; each cycle builds the left-preconditioned
  Arnoldi basis of ``M A`` with one classical Gram-Schmidt projection over
  all basis columns, stops a cycle early only on breakdown
  (``||v|| <= eps * ||M A v_k||``), then solves the Hessenberg least-squares
  problem ('batched': normal equations + Cholesky) or applies Givens rotations
  step by step ('incremental', which also stops a cycle once the rotated
  residual estimate drops below ``ptol = ||M b|| min(1, atol/||b||)``).
* ``tridiagonal_solve``: ``jax.lax.linalg.tridiagonal_solve`` (steppers.py:227)
  for the strictly diagonally dominant column systems of the preconditioner;
  restated as the Thomas algorithm (no pivoting is needed for these systems).
* ``custom_linear_solve``: ``jax.lax.custom_linear_solve`` (steppers.py:483)
  as a torch autograd Function whose backward runs the transpose solve.

Test infrastructure only.
"""

import torch

from . import DTYPE


def tridiagonal_solve(lower, main, upper, rhs):
    """Solve the batched tridiagonal systems along the last axis.

    ``lower[..., 0]`` and ``upper[..., -1]`` are ignored, as in
    ``jax.lax.linalg.tridiagonal_solve``.  Differentiable through autograd.
    """
    n = rhs.shape[-1]
    cp = [None] * n
    dp = [None] * n
    inv = 1.0 / main[..., 0]
    cp[0] = upper[..., 0] * inv
    dp[0] = rhs[..., 0] * inv
    for k in range(1, n):
        den = main[..., k] - lower[..., k] * cp[k - 1]
        inv = 1.0 / den
        cp[k] = upper[..., k] * inv
        dp[k] = (rhs[..., k] - lower[..., k] * dp[k - 1]) * inv
    x = [None] * n
    x[n - 1] = dp[n - 1]
    for k in range(n - 2, -1, -1):
        x[k] = dp[k] - cp[k] * x[k + 1]
    return torch.stack(x, dim=-1)


def _norm(x):
    return torch.sqrt(torch.dot(x, x))


def _safe_normalize(x, thresh=None):
    n = _norm(x)
    if thresh is None:
        thresh = torch.finfo(x.dtype).eps
    use = n > thresh
    if bool(use):
        return x / n, n
    return torch.zeros_like(x), torch.zeros_like(n)


def _arnoldi_step(k, A, M, V, eps):
    """One Arnoldi step: v = M(A(V_k)), one CGS pass, normalise.

    ``V`` is the (restart + 1, n) basis; JAX projects on every column, and
    the columns beyond k are still zero, so projecting on ``V[:k + 1]`` gives
    the same coefficients (zeros for the rest) with a fraction of the work."""
    v = M(A(V[k]))
    v_norm0 = _norm(v)
    Vk = V[:k + 1]
    hk = Vk @ v
    v = v - Vk.T @ hk
    h = torch.zeros(V.shape[0], dtype=v.dtype)
    h[:k + 1] = hk
    unit, vn1 = _safe_normalize(v, thresh=eps * v_norm0)
    return unit, h, vn1


def _lstsq_normal(a, b):
    """``_lstsq``: solve the normal equations with a Cholesky factorisation."""
    a2 = a.T @ a
    b2 = a.T @ b
    L = torch.linalg.cholesky(a2)
    return torch.cholesky_solve(b2[:, None], L)[:, 0]


def gmres(A, b, x0=None, *, tol=1e-5, atol=0.0, restart=20, maxiter=None, M=None,
          solve_method="batched", stats=None):
    """``jax.scipy.sparse.linalg.gmres`` on flat float64 vectors."""
    if x0 is None:
        x0 = torch.zeros_like(b)
    if M is None:
        M = lambda v: v
    size = b.numel()
    if maxiter is None:
        maxiter = 10 * size
    restart = min(restart, size)
    eps = torch.finfo(b.dtype).eps
    b_norm = _norm(b)
    atol = torch.maximum(tol * b_norm, torch.as_tensor(atol, dtype=b.dtype))
    Mb_norm = _norm(M(b))
    ptol = Mb_norm * torch.minimum(torch.ones((), dtype=b.dtype), atol / b_norm)

    x = x0
    unit_r, r_norm = _safe_normalize(M(b - A(x0)))
    k = 0
    arnoldi_steps = 0
    while k < maxiter and bool(r_norm > atol):
        V = torch.zeros(restart + 1, size, dtype=b.dtype)
        V[0] = unit_r
        if solve_method == "batched":
            H = torch.eye(restart, restart + 1, dtype=b.dtype)
            j = 0
            while j < restart:
                unit, h, vn1 = _arnoldi_step(j, A, M, V, eps)
                V[j + 1] = unit
                h = h.clone()
                h[j + 1] = vn1
                H[j, :] = h
                arnoldi_steps += 1
                j += 1
                if bool(vn1 == 0.0):
                    break
            beta = torch.zeros(restart + 1, dtype=b.dtype)
            beta[0] = r_norm
            y = _lstsq_normal(H.T, beta)
        elif solve_method == "incremental":
            R = torch.eye(restart, restart + 1, dtype=b.dtype)
            givens = torch.zeros(restart, 2, dtype=b.dtype)
            beta = torch.zeros(restart + 1, dtype=b.dtype)
            beta[0] = r_norm
            err = r_norm
            j = 0
            while j < restart and bool(err > ptol):
                unit, h, vn1 = _arnoldi_step(j, A, M, V, eps)
                V[j + 1] = unit
                h = h.clone()
                h[j + 1] = vn1
                for i in range(j):  # apply the previous rotations
                    c, s = givens[i, 0], givens[i, 1]
                    h0, h1 = h[i].clone(), h[i + 1].clone()
                    h[i] = c * h0 - s * h1
                    h[i + 1] = s * h0 + c * h1
                hj, hj1 = h[j], h[j + 1]
                denom = torch.sqrt(hj * hj + hj1 * hj1)
                if bool(denom == 0.0):
                    c, s = torch.ones((), dtype=b.dtype), torch.zeros((), dtype=b.dtype)
                else:
                    c, s = hj / denom, -hj1 / denom
                givens[j, 0], givens[j, 1] = c, s
                h[j], h[j + 1] = c * hj - s * hj1, torch.zeros((), dtype=b.dtype)
                R[j, :] = h
                b0, b1 = beta[j].clone(), beta[j + 1].clone()
                beta[j] = c * b0 - s * b1
                beta[j + 1] = s * b0 + c * b1
                err = beta[j + 1].abs()
                arnoldi_steps += 1
                j += 1
            # triangular solve on the j leading columns (rows beyond j unused)
            y = torch.zeros(restart, dtype=b.dtype)
            if j > 0:
                T = R[:j, :j].T
                y[:j] = torch.linalg.solve_triangular(T, beta[:j, None], upper=True)[:, 0]
        else:
            raise ValueError(f"invalid solve_method {solve_method}")
        dx = V[:restart].T @ y
        x = x + dx
        unit_r, r_norm = _safe_normalize(M(b - A(x)))
        k += 1
    if stats is not None:
        stats["cycles"] = k
        stats["arnoldi_steps"] = arnoldi_steps
        stats["residual_norm"] = float(r_norm)
        stats["atol"] = float(atol)
    return x


class _LinearSolve(torch.autograd.Function):
    """``lax.custom_linear_solve(A, b, solve, transpose_solve)`` on flat b.

    Forward returns ``solve(b)``.  Backward maps the solution cotangent
    ``g`` to ``transpose_solve(g)``, the cotangent of ``b``.  Cotangents of
    anything ``solve`` closes over (the initial guess) are not propagated,
    matching custom_linear_solve, which differentiates through ``b`` only.
    """

    @staticmethod
    def forward(ctx, b, solve, transpose_solve):
        ctx.transpose_solve = transpose_solve
        with torch.no_grad():
            return solve(b.detach())

    @staticmethod
    def backward(ctx, g):
        with torch.no_grad():
            return ctx.transpose_solve(g.detach()), None, None


def custom_linear_solve(b, solve, transpose_solve):
    return _LinearSolve.apply(b, solve, transpose_solve)


def linear_transpose(fn, n):
    """Transpose of a linear map on flat float64 vectors of length n via VJP."""
    def fn_T(y):
        x = torch.zeros(n, dtype=DTYPE, requires_grad=True)
        with torch.enable_grad():
            out = fn(x)
            (g,) = torch.autograd.grad(out, x, grad_outputs=y, allow_unused=True)
        return torch.zeros(n, dtype=DTYPE) if g is None else g
    return fn_T
