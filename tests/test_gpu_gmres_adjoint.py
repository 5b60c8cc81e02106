"""The reference's GMRES adjoint study (verification/gmres_adjoint_convergence.py)
on the CUDA path, float64: the trajectory gradient with both solves capped
at `maxiter` restart cycles approaches the tight-tolerance gradient as
`maxiter` grows, a shorter time step (smaller horizontal acoustic Courant
number) gets there in fewer cycles (:1-21), and every series ends below the
study's 1e-6 target (:180-186)."""

import pytest
import torch

import _gmres_adjoint as ga

pytestmark = pytest.mark.gpu

# (dt, maxiter values, maxiter of the reference gradient), subsets of :143-148
SERIES = ((10.0, [2, 4, 8, 15], 100), (2.5, [2, 4], 50), (1.0, [1, 2], 25))


def test_gradient_error_falls_with_maxiter_and_time_step():
    first_below = []
    for dt, iters, ref_it in SERIES:
        _, g0 = ga.gradient(dt, ref_it, 1e-12)
        errs = []
        for it in iters:
            _, gk = ga.gradient(dt, it, 1e-8)
            assert torch.isfinite(gk).all()
            errs.append(float(torch.linalg.vector_norm(gk - g0) / torch.linalg.vector_norm(g0)))
        for a, b in zip(errs[:-1], errs[1:]):
            assert b <= a * 1.01 + 1e-12, (dt, iters, errs)
        assert errs[-1] < 1e-6, (dt, iters, errs)
        first_below.append(next(it for it, e in zip(iters, errs) if e < 1e-4))
    assert first_below == sorted(first_below, reverse=True), first_below
    assert first_below[0] > first_below[-1], first_below
