"""Pins of the float64 CPU oracle against the reference's own known-answer
tests (tests/test_dynamical_core_3d.py, tests/test_core_formula_regressions.py,
tests/test_periodic_boundaries.py) and scipy cross-checks.  CPU only."""

import math

import numpy as np
import pytest
import torch

from _cases import C, build, mountain, shapes5

from oracle.grid import RegionalGrid3D, SleveSimple
from oracle.linalg import tridiagonal_solve
from oracle.ops import CGridOperator3D, map_coordinates_linear, tensor_product_interp_3d
from oracle.steppers import (FluxFormAdvector, SemiImplicitSolver3D, SemiLagrangianAdvector3D, SISLStepper3D)

F64 = torch.float64
NX, NY, NZ, DT = 32, 32, 15, 100.0


@pytest.fixture(scope="module")
def env():
    return build("oracle", NX, NY, NZ, 1000.0, 1000.0, 500.0, h=mountain, dt=DT, N_bv=0.01)


def bgp(ph):
    return ph.precompute_bg(ph.bg_state_ref())


def z(*s):
    return torch.zeros(*s, dtype=F64)


def test_geometry_no_tangling(env):  # test_dynamical_core_3d.py:91-98
    assert float(env[0].dz_m_full.min()) > 0.0


def test_backtracking(env):  # :100-123
    g, op, ph = env
    adv = SemiLagrangianAdvector3D(g, ph, DT)
    st = {"u": torch.ones(NX + 1, NY, NZ, dtype=F64) * 10.0, "v": z(NX, NY + 1, NZ), "eta_dot": z(NX, NY, NZ + 1)}
    dep = adv.compute_departure_indices(st, loc="m", iterations=2)
    X = torch.arange(NX, dtype=F64)[:, None, None]
    err = ((X - dep[0]) - (10.0 * DT / 1000.0) * g.m_factors["m"][..., None]).abs().max()
    assert float(err) < 1e-4


def test_ffsl_mass_conservation(env):  # :125-179
    g, op, ph = env
    bg = bgp(ph)
    rho = ph.bg_state_ref()["rho"]
    st = {"u": torch.ones(NX + 1, NY, NZ, dtype=F64) * 15.0, "v": torch.ones(NX, NY + 1, NZ, dtype=F64) * 5.0,
          "eta_dot": z(NX, NY, NZ + 1)}
    st["u"][0] = 0.0
    st["u"][-1] = 0.0
    st["v"][:, 0] = 0.0
    st["v"][:, -1] = 0.0
    vol = (g.dx * g.dy / g.m_factors["m"][..., None] ** 2) * g.dz_m_full
    m0 = float((rho * vol).sum())
    out = FluxFormAdvector(g, DT).advect_3d_split(rho, st, bg)
    assert abs(float((out * vol).sum()) - m0) / m0 < 1e-14


def test_limiter_prevents_undershoot(env):  # :181-199
    g = env[0]
    X, Y, Zc = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    blob = torch.exp(-((X) ** 2 + (Y) ** 2 + (Zc - 2000.0) ** 2) / (1500.0 ** 2))
    I, J, K = torch.meshgrid(*(torch.arange(n, dtype=F64) for n in (NX, NY, NZ)), indexing="ij")
    coords = torch.stack([I - 0.5, J - 0.5, K - 0.5])
    assert float(tensor_product_interp_3d(blob, coords, use_limiter=False).min()) < 0.0
    assert float(tensor_product_interp_3d(blob, coords, use_limiter=True).min()) >= 0.0


def test_hydrostatic_rest(env):  # :201-228
    g, op, ph = env
    sp = {"u": z(NX + 1, NY, NZ), "v": z(NX, NY + 1, NZ), "w": z(NX, NY, NZ + 1), "pi": z(NX, NY, NZ),
          "eta_dot": z(NX, NY, NZ + 1)}
    assert float(ph.get_tendencies(sp, bgp(ph))["u"].abs().max()) < 1e-4


def test_gmres_manufactured(env):  # :230-280
    g, op, ph = env
    solver = SemiImplicitSolver3D(ph, DT, solver_tol=1e-8, solver_maxiter=100, solver_restart=100)
    gen = torch.Generator().manual_seed(42)
    sh = shapes5(NX, NY, NZ)
    known = {k: torch.rand(sh[k], generator=gen, dtype=F64) * s
             for k, s in (("u", 0.1), ("v", 0.1), ("w", 0.01), ("pi", 0.001), ("eta_dot", 0.001))}
    for k in ("w", "eta_dot"):
        known[k][:, :, 0] = 0.0
        known[k][:, :, -1] = 0.0
    bg = bgp(ph)
    rhs = ph.linear_operator(known, bg, dt=DT, alpha=solver.alpha)
    sol = solver.solve(rhs, bg)
    assert float(solver.relative_residual(sol, rhs, bg)) < 1e-6


def test_kinematic_bottom_preserved(env):  # :335-382
    g, op, ph = env
    bg = bgp(ph)
    rhs = {"u": torch.ones(NX + 1, NY, NZ, dtype=F64) * 10.0, "v": z(NX, NY + 1, NZ), "w": z(NX, NY, NZ + 1),
           "pi": z(NX, NY, NZ), "eta_dot": z(NX, NY, NZ + 1)}
    u_w = op.avg(op.avg(rhs["u"], 0, "u", "m"), 2, "m", "w")
    v_w = op.avg(op.avg(rhs["v"], 1, "v", "m"), 2, "m", "w")
    kb = g.m_factors["w"] * (u_w[:, :, 0] * g.z_xi_w[:, :, 0] + v_w[:, :, 0] * g.z_eta_w[:, :, 0])
    rhs["w"][:, :, 0] = kb
    sol = SemiImplicitSolver3D(ph, DT).solve(rhs, bg)
    assert np.isclose(float(kb.max()), float(sol["w"][:, :, 0].max()), rtol=1e-4)


def _terrain_env():  # :386-406
    def schaer(x, y):
        return 2000.0 * torch.exp(-(x ** 2) / 15000.0 ** 2) * torch.cos(math.pi * x / 8000.0) ** 2
    return build("oracle", 150, 5, 50, 1000.0, 1000.0, 400.0, lat=0.0, h=schaer,
                 transform=SleveSimple(scale_s=4000.0, scale_l=15000.0, n=1.35), dt=DT,
                 damp_height=50 * 400.0, N_bv=0.01)


def test_metric_gradients_terrain():  # :408-425
    g, op, ph = _terrain_env()
    sp = {"u": torch.zeros_like(g.Z_u), "v": torch.zeros_like(g.Z_v), "w": torch.zeros_like(g.Z_w),
          "pi": torch.zeros_like(g.Z_m), "eta_dot": torch.zeros_like(g.Z_w)}
    assert float(ph.get_tendencies(sp, bgp(ph))["u"].abs().max()) <= 1e-6


def test_kinematic_divergence_terrain():  # :427-472
    g, op, ph = _terrain_env()
    bg = bgp(ph)
    u = 10.0 * torch.ones_like(g.Z_u)
    v = torch.zeros_like(g.Z_v)
    m_u, m_v = g.m_factors["u"][..., None], g.m_factors["v"][..., None]
    fx = (u * bg["rho_u"] * bg["th_v_u"] * bg["dz_u"]) / m_u
    fy = (v * bg["rho_v"] * bg["th_v_v"] * bg["dz_v"]) / m_v
    div_h = op.diff(fx, 0, "u", "m") / bg["dz_m_full"] + op.diff(fy, 1, "v", "m") / bg["dz_m_full"]
    fz = torch.cat([torch.zeros(g.nx, g.ny, 1, dtype=F64), torch.cumsum(-div_h * bg["dz_m_full"], dim=2)], dim=2)
    eta = fz / (bg["dz_w_full"] * bg["rho_w"] * bg["th_v_w"])
    sp = {"u": u, "v": v, "w": torch.zeros_like(g.Z_w), "pi": torch.zeros_like(g.Z_m), "eta_dot": eta}
    assert float(ph.get_tendencies(sp, bg)["pi"][:, :, :-1].abs().max()) <= 1e-5


def test_vertical_metric_smoothness():  # :474-483
    g, op, ph = _terrain_env()
    assert float(bgp(ph)["dz_w_full"].min()) >= 10.0


def _rest_state(ph, g):
    return {"u": torch.zeros_like(g.Z_u), "v": torch.zeros_like(g.Z_v), "w": torch.zeros_like(g.Z_w),
            "eta_dot": torch.zeros_like(g.Z_w), "pi": ph.pi_bg, "th_v": ph.theta_bg, "rho": ph.bg_state_ref()["rho"],
            "u_prev": torch.zeros_like(g.Z_u), "v_prev": torch.zeros_like(g.Z_v), "w_prev": torch.zeros_like(g.Z_w),
            "eta_dot_prev": torch.zeros_like(g.Z_w), "tend_th_v_prev": torch.zeros_like(g.Z_m),
            "is_first_step": 1.0}


def test_resting_flat_integration(env):  # :485-507 (50 steps)
    g, op, ph = env
    st = SISLStepper3D(ph, DT)
    s = st.integrate(_rest_state(ph, g), 0.0, 50, None, lambda a, f: a)
    assert float(s["w"].abs().max()) < 1e-7


@pytest.mark.slow
def test_resting_mountain_integration():  # :509-539 (50 steps on a 50x50x40 Agnesi mountain)
    h = lambda x, y: 1500.0 / (1.0 + (x ** 2 + y ** 2) / (30000.0 ** 2))
    g, op, ph = build("oracle", 50, 50, 40, 6000.0, 6000.0, 500.0, lon=5.0, h=h, dt=DT, N_bv=0.01)
    s = SISLStepper3D(ph, DT).integrate(_rest_state(ph, g), 0.0, 50, None, lambda a, f: a)
    assert float(s["w"].abs().max()) < 1e-7


def _small_env(dt, latitude):  # test_core_formula_regressions.py:45-76
    return build("oracle", 8, 8, 5, 2000.0, 2000.0, 500.0, lat=latitude, dt=dt, N_bv=0.0, damp_height=1.0e9,
                 max_damp=0.0, nu_div_factor=0.0, nu_h_factor=0.0)


def _base(ph, g, u=0.0, v=0.0):
    s = _rest_state(ph, g)
    s["u"] = torch.full_like(g.Z_u, u)
    s["v"] = torch.full_like(g.Z_v, v)
    for k in ("u_prev", "v_prev", "w_prev", "eta_dot_prev", "tend_th_v_prev", "is_first_step"):
        s.pop(k)
    return s


def test_nonlinear_pgf_does_not_rescale_coriolis():  # test_core_formula_regressions.py:168-194
    def advance(off):
        g, op, ph = _small_env(0.05, 55.0)
        s = _base(ph, g, 8.0, 12.0)
        s["th_v"] = s["th_v"] + off
        s["rho"] = C["p0"] / (C["Rd"] * s["th_v"]) * s["pi"] ** (C["cvd"] / C["Rd"])
        st = SISLStepper3D(ph, 0.05, alpha=0.5, solver_tol=1e-11, solver_maxiter=80, solver_restart=40)
        return st.step(s, 0.0, None, lambda a, f: a)
    ref, warm = advance(0.0), advance(30.0)
    err = max(float((warm["u"][1:-1] - ref["u"][1:-1]).abs().max()),
              float((warm["v"][:, 1:-1] - ref["v"][:, 1:-1]).abs().max()))
    cor = float((ref["u"] - 8.0).abs().max())
    assert cor > 1e-8
    assert err < 1e-5 * cor


def test_full_metric_curvature_tendency():  # test_core_formula_regressions.py:197-235
    dt = 1.0e-3
    g, op, ph = _small_env(dt, 0.0)
    for loc in ("m", "u", "v", "w"):
        g.m_factors[loc] = torch.ones_like(g.m_factors[loc])
    op.m_factors = {loc: m[..., None] for loc, m in g.m_factors.items()}
    g.f_u = torch.zeros_like(g.f_u)
    g.f_v = torch.zeros_like(g.f_v)
    g.dm_dx_m = torch.full_like(g.dm_dx_m, 2.0e-4)
    g.dm_dy_m = torch.full_like(g.dm_dy_m, -1.0e-4)
    s = _base(ph, g, 10.0, 6.0)
    thp = s["th_v"] - ph.theta_bg
    prime = {"u": s["u"], "v": s["v"], "w": s["w"], "eta_dot": s["eta_dot"], "pi": s["pi"] - ph.pi_bg,
             "th_v": s["th_v"], "th_v_prime_u": op.avg(thp, 0, "m", "u"), "th_v_prime_v": op.avg(thp, 1, "m", "v"),
             "th_v_prime_w": op.avg(thp, 2, "m", "w")}
    exp = ph.get_tendencies(prime, bgp(ph), is_explicit=True)
    res = SISLStepper3D(ph, dt, alpha=0.5, solver_tol=1e-12, solver_maxiter=80, solver_restart=40).step(
        s, 0.0, None, lambda a, f: a)
    eu = float(((res["u"] - s["u"]) / dt - exp["u"])[1:-1].abs().max())
    ev = float(((res["v"] - s["v"]) / dt - exp["v"])[:, 1:-1].abs().max())
    sig = max(float(exp["u"].abs().max()), float(exp["v"].abs().max()))
    assert sig > 1e-4
    assert max(eu, ev) < 2e-3 * sig


def test_closed_box_density_conserved():  # test_core_formula_regressions.py:238-292 (density part)
    g, op, ph = _small_env(0.02, 45.0)
    s = _base(ph, g)
    iu = torch.arange(g.nx + 1, dtype=F64)[:, None, None]
    jv = torch.arange(g.ny + 1, dtype=F64)[None, :, None]
    s["u"] = 2.0 * torch.sin(math.pi * iu / g.nx) + torch.zeros_like(s["u"])
    s["v"] = -1.5 * torch.sin(math.pi * jv / g.ny) + torch.zeros_like(s["v"])
    vol = g.dx * g.dy * g.dz_m_full / g.m_factors["m"][..., None] ** 2
    m0 = float((s["rho"] * vol).sum())
    res = SISLStepper3D(ph, 0.02, alpha=0.5, solver_tol=1e-11, solver_maxiter=80, solver_restart=40).step(
        s, 0.0, None, lambda a, f: a)
    assert abs(float((res["rho"] * vol).sum()) - m0) / m0 < 1e-10


def test_periodic_operators():  # tests/test_periodic_boundaries.py:19-48
    g = RegionalGrid3D(8, 4, 2, 1.0, 1.0, 1.0, 0.0, 0.0)
    op = CGridOperator3D(g, periodic_axes=(0,))
    f = torch.arange(8, dtype=F64)[:, None, None]
    d = op.diff(f, 0, "m", "u")[:, 0, 0]
    a = op.avg(f, 0, "m", "u")[:, 0, 0]
    assert torch.allclose(d[[0, -1]], torch.tensor(-7.0, dtype=F64))
    assert torch.allclose(a[[0, -1]], torch.tensor(3.5, dtype=F64))
    assert torch.allclose(d[1:-1], torch.ones(7, dtype=F64))
    d0 = CGridOperator3D(g).diff(f, 0, "m", "u")[:, 0, 0]
    assert torch.allclose(d0[[0, -1]], torch.ones(2, dtype=F64))


def test_periodic_ffsl():  # tests/test_periodic_boundaries.py:51-82
    g = RegionalGrid3D(8, 4, 2, 1.0, 1.0, 1.0, 0.0, 0.0)
    adv = FluxFormAdvector(g, dt=1.0, periodic_axes=(0,))
    s = torch.tensor([1.0, 2.0, 4.0, 8.0, 16.0, 32.0, 64.0, 128.0], dtype=F64)
    assert torch.allclose(adv.advect_1d(s, torch.ones(9, dtype=F64), periodic=True), torch.roll(s, 1))
    assert torch.allclose(adv.advect_1d(s, -torch.ones(9, dtype=F64), periodic=True), torch.roll(s, -1))
    s2 = torch.tensor([0.0, 0.0, 1.0, 2.0, 1.0, 0.0, 0.0, 0.0], dtype=F64)
    t = adv.advect_1d(s2, torch.full((9,), 0.35, dtype=F64), periodic=True)
    assert abs(float(t.sum()) - float(s2.sum())) < 1e-12 and float(t.min()) >= 0.0


def test_trilinear_matches_scipy():
    from scipy.ndimage import map_coordinates
    gen = torch.Generator().manual_seed(1)
    f = torch.randn(7, 6, 5, generator=gen, dtype=F64)
    coords = torch.stack([torch.rand((4, 3, 2), generator=gen, dtype=F64) * (n + 2) - 1 for n in f.shape])
    ref = map_coordinates(f.numpy(), coords.numpy(), order=1, mode="nearest")
    assert np.max(np.abs(map_coordinates_linear(f, coords).numpy() - ref)) < 1e-13


def test_thomas_matches_scipy_banded():
    from scipy.linalg import solve_banded
    gen = torch.Generator().manual_seed(2)
    n = 12
    lo = -torch.rand(n, generator=gen, dtype=F64)
    up = -torch.rand(n, generator=gen, dtype=F64)
    lo[0] = 0.0
    up[-1] = 0.0
    main = 1.0 - lo - up
    b = torch.randn(n, generator=gen, dtype=F64)
    ab = np.zeros((3, n))
    ab[0, 1:] = up[:-1].numpy()
    ab[1] = main.numpy()
    ab[2, :-1] = lo[1:].numpy()
    ref = solve_banded((1, 1), ab, b.numpy())
    assert np.max(np.abs(tridiagonal_solve(lo, main, up, b).numpy() - ref)) < 1e-13


def test_ffsl_clip_tie_passes_half_the_cotangent():
    """jnp.clip (steppers.py:589) is maximum then minimum, whose gradient
    splits an exact tie: a wall interface at rest (departure point exactly
    0) passes half the Courant-number cotangent."""
    adv = FluxFormAdvector(RegionalGrid3D(4, 4, 4, 1.0, 1.0, 1.0, 0.0, 0.0), 1.0)
    s = torch.tensor([[1.0, 2.0, 4.0]], dtype=F64)
    c = torch.zeros(1, 4, dtype=F64, requires_grad=True)
    out = adv._advect_last(s, c, False)
    (g,) = torch.autograd.grad(out[0, 0], c)
    # out[0] = Md(1) - Md(0); Md(0) at the tie dep = 0 has slope M(1) - M(0) = s[0]
    assert float(g[0, 0]) == pytest.approx(0.5 * float(s[0, 0]))
    assert float(g[0, 1]) == pytest.approx(-float(s[0, 1]))


def _sine(x, y, z, lx, ly, lz):
    return torch.sin(2 * math.pi * x / lx) * torch.cos(2 * math.pi * y / ly) * torch.sin(2 * math.pi * z / lz)


def test_tricubic_convergence_order():
    """verification/sisl_component_convergence.py:53-90: interpolating a sine
    field at a fixed fractional offset converges at order 3-4."""
    errs = []
    for N in (16, 32, 64):
        lx = 10000.0
        dx = lx / N
        g = RegionalGrid3D(N, N, N, dx, dx, dx, 0.0, 0.0)
        X, Y, Z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
        Xt, Yt, Zt = X + 0.37 * dx, Y + 0.23 * dx, Z + 0.45 * dx
        co = torch.stack([(Xt + lx / 2) / dx - 0.5, (Yt + lx / 2) / dx - 0.5, Zt / dx - 0.5])
        out = tensor_product_interp_3d(_sine(X, Y, Z, lx, lx, lx), co)
        ex, m = _sine(Xt, Yt, Zt, lx, lx, lx), N // 4
        errs.append(float(torch.sqrt(torch.mean((out - ex)[m:-m, m:-m, m:-m] ** 2))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(2.8 < r < 4.2 for r in rates), (errs, rates)


def test_trajectory_convergence_order():
    """verification/sisl_component_convergence.py:147-197: the midpoint
    departure points of the strain flow u = a x against the exact
    characteristic x exp(-a dt) converge at local order 3."""
    r, L, Lz, a = 64, 2.0e6, 1.0e4, 1.0e-4
    dx = L / r
    g = RegionalGrid3D(r, r, r, dx, dx, Lz / r, 0.0, 0.0)
    for k in g.m_factors:
        g.m_factors[k] = torch.ones_like(g.m_factors[k])
    ph = build_physics(g)
    Xu, _, _ = torch.meshgrid(g.x_c, g.y_m, g.z_m, indexing="ij")
    Xm, _, _ = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    st = {"u": a * Xu, "v": z(r, r + 1, r), "w": z(r, r, r + 1), "eta_dot": z(r, r, r + 1)}
    errs = []
    for dt in (400.0, 200.0, 100.0, 50.0):
        c = SemiLagrangianAdvector3D(g, ph, dt).compute_departure_indices(st, loc="m", iterations=8)
        ex, m = (Xm * math.exp(-a * dt) + L / 2) / dx - 0.5, r // 4
        errs.append(dx * float(torch.sqrt(torch.mean((c[0] - ex)[m:-m, m:-m, m:-m] ** 2))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(3)]
    assert all(2.8 < q < 3.2 for q in rates), (errs, rates)


def build_physics(g):
    from oracle.euler import Euler3D
    return Euler3D(g, CGridOperator3D(g), C, dt=1.0)


@pytest.mark.parametrize("r", [8, 16])
def test_gmres_inversion_sweep(r):
    """verification/sisl_component_convergence.py:203-260: the preconditioned
    GMRES (tol 1e-12, the solver's default restart 20 / maxiter 20) inverts
    the Helmholtz operator of a 60N grid to relative residual < 1e-9."""
    from oracle.euler import Euler3D
    L, Lz, dt = 2.0e6, 1.0e4, 60.0
    g = RegionalGrid3D(r, r, r, L / r, L / r, Lz / r, 60.0, 30.0)
    ph = Euler3D(g, CGridOperator3D(g), C, dt=dt, N_bv=0.01)
    sol = SemiImplicitSolver3D(ph, dt, alpha=0.55, solver_tol=1e-12)
    gen = torch.Generator().manual_seed(42)
    U = lambda *s: torch.rand(*s, generator=gen, dtype=F64)
    x = {"u": U(r + 1, r, r) * 5.0, "v": U(r, r + 1, r) * 5.0, "w": U(r, r, r + 1) * 0.1,
         "pi": U(r, r, r) * 0.001, "eta_dot": U(r, r, r + 1) * 0.001}
    for k in ("w", "eta_dot"):
        x[k][:, :, 0] = 0.0
        x[k][:, :, -1] = 0.0
    bg = bgp(ph)
    rhs = ph.linear_operator(x, bg, dt, alpha=0.55)
    xn = sol.solve(rhs, bg)
    assert float(sol.relative_residual(xn, rhs, bg)) < 1e-9


# ---------------------------------------------------------------------------
# Split-explicit oracle (oracle/split_explicit.py) pinned to the reference's
# own split-explicit tests (tests/test_core_formula_regressions.py): the
# Exner slow forcing carries the theta' flux (:130-166) and a complete step
# keeps the closed-box density and passive-tracer budgets through the final
# EOS and tracer reconciliation (:238-292), on their 8x8x5 flat box.
# ---------------------------------------------------------------------------

def _split_env(dt, suite=None):
    from oracle.grid import RegionalGrid3D
    from oracle.ops import CGridOperator3D
    from oracle.euler import Euler3D
    g = RegionalGrid3D(8, 8, 5, 2000.0, 2000.0, 500.0, 45.0, 0.0, h_func=lambda x, y: 0.0 * (x + y))
    op = CGridOperator3D(g)
    ph = Euler3D(g, op, C, dt=dt, N_bv=0.0, damp_height=1e9, max_damp=0.0, nu_div_factor=0.0, nu_h_factor=0.0,
                 physics_suite=suite)
    return g, op, ph


def _split_base(ph, g):
    z = lambda *s: torch.zeros(*s, dtype=torch.float64)
    rho = C["p0"] / (C["Rd"] * ph.theta_bg) * ph.pi_bg ** (C["cvd"] / C["Rd"])
    return {"u": z(g.nx + 1, g.ny, g.nz), "v": z(g.nx, g.ny + 1, g.nz), "w": z(g.nx, g.ny, g.nz + 1),
            "eta_dot": z(g.nx, g.ny, g.nz + 1), "pi": ph.pi_bg.clone(), "th_v": ph.theta_bg.clone(), "rho": rho}


def test_split_oracle_continuity_includes_theta_prime_flux():
    from oracle.split_explicit import SplitExplicitStepper3D
    g, op, ph = _split_env(0.2)
    st = SplitExplicitStepper3D(ph, dt=0.2, ns=2, alpha=0.5)
    s = _split_base(ph, g)
    x = torch.arange(g.nx + 1, dtype=torch.float64)[:, None, None]
    zz = torch.arange(g.nz, dtype=torch.float64)[None, None, :]
    s["u"] = 3.0 + 0.15 * x + torch.zeros_like(s["u"])
    thp = 4.0 + 0.3 * torch.arange(g.nx, dtype=torch.float64)[:, None, None] + 0.2 * zz + torch.zeros_like(s["th_v"])
    s["th_v"] = ph.theta_bg + thp
    s["rho"] = C["p0"] / (C["Rd"] * s["th_v"]) * s["pi"] ** (C["cvd"] / C["Rd"])
    bg = st._bg()
    actual = st._compute_slow_tendencies(s, bg, {}, {}, None)["pi"]
    prime = {"u": s["u"], "v": s["v"], "w": s["w"], "eta_dot": s["eta_dot"], "pi": s["pi"] - ph.pi_bg,
             "th_v": s["th_v"], "th_v_prime_u": op.avg(thp, 0, "m", "u"), "th_v_prime_v": op.avg(thp, 1, "m", "v"),
             "th_v_prime_w": op.avg(thp, 2, "m", "w")}
    linear = ph.get_tendencies(prime, bg, is_explicit=True)["pi"]
    nonlinear = ph.nonlinear_pi_tendency(prime, thp, bg)
    err = float((actual - (linear + nonlinear)).abs().max())
    sig = float(nonlinear.abs().max())
    assert sig > 1e-12 and err < 1e-11 * sig


def test_split_oracle_conserves_density_and_tracer_mass():
    from oracle.split_explicit import SplitExplicitStepper3D

    class Tracer:
        tracer_keys = ["q_test"]

        def get_explicit_tendencies(self, state, bg, interior_mask=None, ml_params=None):
            return {}

        def apply_state_updates(self, state):
            return state

    dt = 0.02
    g, op, ph = _split_env(dt, Tracer())
    s = _split_base(ph, g)
    iu = torch.arange(g.nx + 1, dtype=torch.float64)[:, None, None]
    jv = torch.arange(g.ny + 1, dtype=torch.float64)[None, :, None]
    s["u"] = 2.0 * torch.sin(math.pi * iu / g.nx) + torch.zeros_like(s["u"])
    s["v"] = -1.5 * torch.sin(math.pi * jv / g.ny) + torch.zeros_like(s["v"])
    x = torch.arange(g.nx, dtype=torch.float64)[:, None, None]
    y = torch.arange(g.ny, dtype=torch.float64)[None, :, None]
    s["q_test"] = 1.0 + 0.2 * torch.sin(2 * math.pi * x / g.nx) * torch.cos(2 * math.pi * y / g.ny) \
        + torch.zeros_like(s["rho"])
    vol = g.dx * g.dy * g.dz_m_full / g.m_factors["m"][..., None] ** 2
    m0 = float((s["rho"] * vol).sum())
    t0 = float((s["rho"] * s["q_test"] * vol).sum())
    st = SplitExplicitStepper3D(ph, dt, ns=2, alpha=0.5)
    moved = st.ffsl_advector.advect_3d_split(s["rho"] * s["q_test"], s, st._bg())
    r = st.step(dict(s), 0.0, None, lambda a, f: a)
    assert abs(float((r["rho"] * vol).sum()) - m0) / m0 < 1e-10
    assert abs(float((r["rho"] * r["q_test"] * vol).sum()) - t0) / t0 < 1e-10
    assert float(torch.linalg.norm(r["rho"] * r["q_test"] - moved) / torch.linalg.norm(moved)) < 1e-12
