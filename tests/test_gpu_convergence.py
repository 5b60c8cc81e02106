"""The reference's component convergence verification
(verification/sisl_component_convergence.py) on the CUDA kernels, float64:
tricubic interpolation order 3-4 (unit 1), midpoint trajectory local order 3
(unit 3), and the preconditioned GMRES inverting the Helmholtz operator to
relative residual < 1e-9 at N = 8 ... 64 (unit 4)."""

import math

import pytest
import torch

from _cases import C

pytestmark = pytest.mark.gpu
F64 = torch.float64


def _sine(x, y, z, lx):
    return torch.sin(2 * math.pi * x / lx) * torch.cos(2 * math.pi * y / lx) * torch.sin(2 * math.pi * z / lx)


def test_tricubic_convergence_order_cuda():
    from suetes_b200 import RegionalGrid3D, tensor_product_interp_3d
    errs = []
    for N in (16, 32, 64):
        lx = 10000.0
        dx = lx / N
        g = RegionalGrid3D(N, N, N, dx, dx, dx, 0.0, 0.0, device="cuda")
        X, Y, Z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
        Xt, Yt, Zt = X + 0.37 * dx, Y + 0.23 * dx, Z + 0.45 * dx
        co = torch.stack([(Xt + lx / 2) / dx - 0.5, (Yt + lx / 2) / dx - 0.5, Zt / dx - 0.5])
        out = tensor_product_interp_3d(_sine(X, Y, Z, lx), co)
        m = N // 4
        errs.append(float(torch.sqrt(torch.mean((out - _sine(Xt, Yt, Zt, lx))[m:-m, m:-m, m:-m] ** 2))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(2.8 < r < 4.2 for r in rates), (errs, rates)


def test_trajectory_convergence_order_cuda():
    from suetes_b200 import CGridOperator3D, Euler3D, RegionalGrid3D, SemiLagrangianAdvector3D
    r, L, Lz, a = 64, 2.0e6, 1.0e4, 1.0e-4
    dx = L / r
    g = RegionalGrid3D(r, r, r, dx, dx, Lz / r, 0.0, 0.0, device="cuda")
    for k in g.m_factors:
        g.m_factors[k] = torch.ones_like(g.m_factors[k])
    ph = Euler3D(g, CGridOperator3D(g), C, dt=1.0)
    Xu, _, _ = torch.meshgrid(g.x_c, g.y_m, g.z_m, indexing="ij")
    Xm, _, _ = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    z = lambda *s: torch.zeros(*s, dtype=F64, device="cuda")
    st = {"u": a * Xu, "v": z(r, r + 1, r), "w": z(r, r, r + 1), "eta_dot": z(r, r, r + 1)}
    errs = []
    for dt in (400.0, 200.0, 100.0, 50.0):
        c = SemiLagrangianAdvector3D(g, ph, dt).compute_departure_indices(st, loc="m", iterations=8)
        ex, m = (Xm * math.exp(-a * dt) + L / 2) / dx - 0.5, r // 4
        errs.append(dx * float(torch.sqrt(torch.mean((c[0] - ex)[m:-m, m:-m, m:-m] ** 2))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(3)]
    assert all(2.8 < q < 3.2 for q in rates), (errs, rates)


@pytest.mark.parametrize("r", [8, 16, 32, 64])
def test_gmres_inversion_sweep_cuda(r):
    from suetes_b200 import CGridOperator3D, Euler3D, RegionalGrid3D, SemiImplicitSolver3D
    L, Lz, dt = 2.0e6, 1.0e4, 60.0
    g = RegionalGrid3D(r, r, r, L / r, L / r, Lz / r, 60.0, 30.0, device="cuda")
    ph = Euler3D(g, CGridOperator3D(g), C, dt=dt, N_bv=0.01)
    sol = SemiImplicitSolver3D(ph, dt, alpha=0.55, solver_tol=1e-12)
    gen = torch.Generator().manual_seed(42)
    U = lambda *s: torch.rand(*s, generator=gen, dtype=F64)
    x = {"u": U(r + 1, r, r) * 5.0, "v": U(r, r + 1, r) * 5.0, "w": U(r, r, r + 1) * 0.1,
         "pi": U(r, r, r) * 0.001, "eta_dot": U(r, r, r + 1) * 0.001}
    for k in ("w", "eta_dot"):
        x[k][:, :, 0] = 0.0
        x[k][:, :, -1] = 0.0
    x = {k: v.cuda() for k, v in x.items()}
    bg = ph.precompute_bg(ph.bg_state_ref())
    rhs = ph.linear_operator(x, bg, dt, alpha=0.55)
    xn = sol.solve(rhs, bg)
    assert float(sol.relative_residual(xn, rhs, bg)) < 1e-9
