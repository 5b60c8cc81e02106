"""CUDA kernels vs the float64 CPU oracle on identical seeded inputs.

Tolerances: float64 kernels agree with the oracle to round-off (relative L2
<= 1e-11 for stencils and interpolation; GMRES solutions to the solver
tolerance); float32 kernels to relative L2 <= 2e-5 per field.
"""

import math

import pytest
import torch

from _cases import C, build, max_abs, mountain, random_fields, rel_l2, shapes5, to_cpu, to_cuda

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 15
SCALES = {"u": 0.1, "v": 0.1, "w": 0.01, "pi": 1e-3, "eta_dot": 1e-3}
TOL = {torch.float64: 1e-11, torch.float32: 2e-5}


@pytest.fixture(scope="module")
def mountain_pair():
    o = build("oracle", NX, NY, NZ, 1000.0, 1000.0, 500.0, h=mountain, dt=100.0, N_bv=0.01)
    p = build("cuda", NX, NY, NZ, 1000.0, 1000.0, 500.0, h=mountain, device="cuda", dt=100.0, N_bv=0.01)
    return o, p


def _bg(ph):
    return ph.precompute_bg(ph.bg_state_ref())


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_linear_operator(mountain_pair, dtype):
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    x = random_fields(shapes5(NX, NY, NZ), 7, SCALES)
    ref = oph.linear_operator(x, _bg(oph), 100.0, alpha=0.55)
    out = pph.linear_operator(to_cuda(x, dtype), _bg(pph), 100.0, alpha=0.55)
    for k in ref:
        assert rel_l2(out[k], ref[k]) < TOL[dtype], (k, rel_l2(out[k], ref[k]))


@pytest.mark.parametrize("periodic", [(0,), (0, 1)])
def test_linear_operator_periodic(periodic):
    o = build("oracle", 12, 10, 6, 2000.0, 2000.0, 500.0, h=mountain, periodic=periodic, dt=30.0)
    p = build("cuda", 12, 10, 6, 2000.0, 2000.0, 500.0, h=mountain, periodic=periodic, device="cuda", dt=30.0)
    x = random_fields(shapes5(12, 10, 6), 3, SCALES)
    ref = o[2].linear_operator(x, _bg(o[2]), 30.0, alpha=0.5)
    out = p[2].linear_operator(to_cuda(x), _bg(p[2]), 30.0, alpha=0.5)
    for k in ref:
        assert rel_l2(out[k], ref[k]) < 1e-11, k


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_preconditioner(mountain_pair, dtype):
    from oracle.steppers import VerticalPreconditioner as OP
    from suetes_b200 import VerticalPreconditioner as PP
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    r = random_fields(shapes5(NX, NY, NZ), 11, {"u": 0.1, "v": 0.1, "w": 0.01, "pi": 1.0, "eta_dot": 0.1})
    om = OP(oph, 100.0, alpha=0.55)
    om.precompute_banded(_bg(oph))
    pm = PP(pph, 100.0, alpha=0.55)
    pm.precompute_banded(_bg(pph))
    ref = om(r)
    out = pm(to_cuda(r, dtype))
    for k in ref:
        assert rel_l2(out[k], ref[k]) < TOL[dtype] * (10 if dtype == torch.float32 else 1), (k, rel_l2(out[k], ref[k]))


@pytest.mark.parametrize("limiter", [False, True])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_tricubic(dtype, limiter):
    from oracle.ops import tensor_product_interp_3d as ref_interp
    from suetes_b200 import tensor_product_interp_3d
    gen = torch.Generator().manual_seed(5)
    f = torch.randn(17, 13, 9, generator=gen, dtype=torch.float64)
    shape = (11, 7, 5)
    coords = torch.stack([torch.rand(shape, generator=gen, dtype=torch.float64) * (n + 4) - 2
                          for n in f.shape])  # includes points outside the field
    ref = ref_interp(f, coords, use_limiter=limiter)
    out = tensor_product_interp_3d(f.to("cuda", dtype), coords.to("cuda", dtype), use_limiter=limiter)
    assert tuple(out.shape) == shape
    assert rel_l2(out, ref) < (1e-13 if dtype == torch.float64 else 2e-6)


def test_trilinear_matches_scipy():
    import numpy as np
    from scipy.ndimage import map_coordinates
    from suetes_b200 import map_coordinates_linear
    gen = torch.Generator().manual_seed(9)
    f = torch.randn(9, 8, 7, generator=gen, dtype=torch.float64)
    coords = torch.stack([torch.rand((6, 5, 4), generator=gen, dtype=torch.float64) * (n + 2) - 1 for n in f.shape])
    ref = map_coordinates(f.numpy(), coords.numpy(), order=1, mode="nearest")
    out = map_coordinates_linear(f.cuda(), coords.cuda()).cpu().numpy()
    assert np.max(np.abs(out - ref)) < 1e-13


@pytest.mark.parametrize("loc", ["m", "u", "v", "w"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_departure_points(mountain_pair, loc, dtype):
    from oracle.steppers import SemiLagrangianAdvector3D as OA
    from suetes_b200 import SemiLagrangianAdvector3D as PA
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    s = random_fields({"u": (NX + 1, NY, NZ), "v": (NX, NY + 1, NZ), "eta_dot": (NX, NY, NZ + 1)}, 21,
                      {"u": 15.0, "v": 15.0, "eta_dot": 0.01})
    ref = OA(og, oph, 100.0).compute_departure_indices(s, loc=loc)
    out = PA(pg, pph, 100.0).compute_departure_indices(to_cuda(s, dtype), loc=loc)
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    assert max_abs(out, ref) < tol, max_abs(out, ref)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_explicit_tendencies(dtype):
    o = build("oracle", 16, 14, 10, 1000.0, 1000.0, 500.0, h=mountain, dt=20.0, N_bv=0.01, nu_h_factor=0.1)
    p = build("cuda", 16, 14, 10, 1000.0, 1000.0, 500.0, h=mountain, device="cuda", dt=20.0, N_bv=0.01,
              nu_h_factor=0.1)
    oph, pph = o[2], p[2]
    x = random_fields(shapes5(16, 14, 10), 13, {"u": 5.0, "v": 5.0, "w": 0.5, "pi": 1e-3, "eta_dot": 1e-3})
    gen = torch.Generator().manual_seed(14)
    thp = torch.randn(16, 14, 10, generator=gen, dtype=torch.float64)
    obg = _bg(oph)
    sp = dict(x)
    sp["th_v"] = oph.theta_bg + thp
    sp["th_v_prime_u"] = oph.op.avg(thp, 0, "m", "u")
    sp["th_v_prime_v"] = oph.op.avg(thp, 1, "m", "v")
    sp["th_v_prime_w"] = oph.op.avg(thp, 2, "m", "w")
    ref = oph.get_tendencies(sp, obg, True)
    psp = to_cuda(x, dtype)
    psp["th_v"] = (pph.theta_bg + thp.cuda()).to(dtype)
    if dtype == torch.float32:  # pass the perturbation itself to avoid float32 cancellation
        psp.pop("th_v")
        psp["th_v_prime_m"] = thp.to("cuda", dtype)
    out = pph.get_tendencies(psp, _bg(pph), True)
    tol = 1e-10 if dtype == torch.float64 else 5e-5
    for k in ("u", "v", "w", "pi", "th_v", "phys_diff_u", "phys_diff_v", "phys_diff_w", "phys_diff_th_v"):
        assert rel_l2(out[k], ref[k]) < tol, (k, rel_l2(out[k], ref[k]))
    nl_ref = oph.nonlinear_pi_tendency(x, thp, obg)
    nl = pph.nonlinear_pi_tendency(to_cuda(x, dtype), thp.to("cuda", dtype), _bg(pph))
    assert rel_l2(nl, nl_ref) < tol


def test_linear_tendencies(mountain_pair):
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    x = random_fields(shapes5(NX, NY, NZ), 17, SCALES)
    ref = oph.get_tendencies(x, _bg(oph), False)
    out = pph.get_tendencies(to_cuda(x), _bg(pph), False)
    for k in ("u", "v", "w", "pi", "th_v"):
        assert rel_l2(out[k], ref[k]) < 1e-11, k


@pytest.mark.parametrize("method", ["batched", "incremental"])
def test_gmres_manufactured_solution(mountain_pair, method):
    """tests/test_dynamical_core_3d.py:230-280 on the CUDA solver."""
    from suetes_b200 import SemiImplicitSolver3D
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    gen = torch.Generator().manual_seed(42)
    sh = shapes5(NX, NY, NZ)
    known = {k: torch.rand(sh[k], generator=gen, dtype=torch.float64) * s
             for k, s in (("u", 0.1), ("v", 0.1), ("w", 0.01), ("pi", 0.001), ("eta_dot", 0.001))}
    for k in ("w", "eta_dot"):
        known[k][:, :, 0] = 0.0
        known[k][:, :, -1] = 0.0
    bg = _bg(pph)
    solver = SemiImplicitSolver3D(pph, 100.0, solver_tol=1e-8, solver_maxiter=100, solver_restart=100,
                                  solve_method=method)
    rhs = pph.linear_operator(to_cuda(known), bg, dt=100.0, alpha=solver.alpha)
    sol = solver.solve(rhs, bg)
    rr = float(solver.relative_residual(sol, rhs, bg))
    assert all(torch.isfinite(v).all() for v in sol.values())
    assert rr < 1e-6, (rr, solver.last_info)
    assert solver.last_info["converged"]
    for k in known:
        assert rel_l2(sol[k], known[k]) < 1e-3, k


def test_gmres_matches_oracle_small():
    """Same solve on both sides (batched, identical settings)."""
    from oracle.steppers import SemiImplicitSolver3D as OS
    from suetes_b200 import SemiImplicitSolver3D as PS
    o = build("oracle", 10, 8, 6, 2000.0, 2000.0, 500.0, h=mountain, dt=20.0)
    p = build("cuda", 10, 8, 6, 2000.0, 2000.0, 500.0, h=mountain, device="cuda", dt=20.0)
    rhs = random_fields(shapes5(10, 8, 6), 99, SCALES)
    for k in ("w", "eta_dot"):
        rhs[k][:, :, 0] = 0.0
        rhs[k][:, :, -1] = 0.0
    x0 = random_fields(shapes5(10, 8, 6), 98, SCALES)
    os_ = OS(o[2], 20.0, solver_tol=1e-10, solver_maxiter=40, solver_restart=15)
    ps_ = PS(p[2], 20.0, solver_tol=1e-10, solver_maxiter=40, solver_restart=15)
    ref = os_.solve(rhs, _bg(o[2]), x0=x0)
    out = ps_.solve(to_cuda(rhs), _bg(p[2]), x0=to_cuda(x0))
    assert ps_.last_info["cycles"] == os_.last_stats["forward"]["cycles"]
    for k in ref:
        assert rel_l2(out[k], ref[k]) < 1e-8, (k, rel_l2(out[k], ref[k]))


def _bubble_state(ph, g, amp=2.0, r0=1000.0, zc=1500.0):
    th = ph.theta_bg
    x, y, z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    r = torch.sqrt(x ** 2 + y ** 2 + (z - zc) ** 2)
    th = th + torch.where(r < r0, amp * torch.cos(0.5 * math.pi * r / r0) ** 2, torch.zeros_like(r))
    rho = C["p0"] / (C["Rd"] * th) * ph.pi_bg ** (C["cvd"] / C["Rd"])
    z3 = lambda *s: torch.zeros(*s, dtype=torch.float64, device=th.device)
    nx, ny, nz = g.nx, g.ny, g.nz
    return {"u": z3(nx + 1, ny, nz) + 3.0, "v": z3(nx, ny + 1, nz) - 2.0, "w": z3(nx, ny, nz + 1),
            "eta_dot": z3(nx, ny, nz + 1), "pi": ph.pi_bg.clone(), "th_v": th, "rho": rho}


@pytest.mark.parametrize("method", ["batched", "incremental"])
def test_step_matches_oracle(method):
    """Two full SISL steps (mountain, bubble, winds, hyperdiffusion, divergence damping)."""
    from oracle.steppers import SISLStepper3D as OSt
    from suetes_b200 import SISLStepper3D as PSt
    kw = dict(dt=10.0, N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1, damp_height=4000.0, max_damp=0.5)
    o = build("oracle", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, **kw)
    p = build("cuda", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, device="cuda", **kw)
    os_ = OSt(o[2], 10.0, alpha=0.55, solver_tol=1e-12, solver_maxiter=60, solver_restart=30, solve_method=method)
    ps_ = PSt(p[2], 10.0, alpha=0.55, solver_tol=1e-12, solver_maxiter=60, solver_restart=30, solve_method=method)
    so = _bubble_state(o[2], o[0])
    sp = to_cuda(to_cpu(_bubble_state(o[2], o[0])))
    ident = lambda s, f: s
    for n in range(2):
        so = os_.step(so, n * 10.0, None, ident)
        sp = ps_.step(sp, n * 10.0, None, ident)
    for k in ("u", "v", "w", "eta_dot", "rho", "u_prev", "eta_dot_prev", "tend_th_v_prev"):
        assert rel_l2(sp[k], so[k]) < 1e-8, (k, rel_l2(sp[k], so[k]))
    for k, bg in (("pi", o[2].pi_bg), ("th_v", o[2].theta_bg)):
        assert rel_l2(sp[k].double().cpu() - bg, so[k] - bg) < 1e-8, k


def test_step_float32_close_to_oracle():
    from oracle.steppers import SISLStepper3D as OSt
    from suetes_b200 import SISLStepper3D as PSt
    kw = dict(dt=10.0, N_bv=0.01, nu_h_factor=0.0, nu_div_factor=0.0)
    o = build("oracle", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, **kw)
    p = build("cuda", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, device="cuda", **kw)
    os_ = OSt(o[2], 10.0, solver_tol=1e-12, solver_maxiter=60, solver_restart=30)
    ps_ = PSt(p[2], 10.0, solver_tol=1e-6, solver_maxiter=60, solver_restart=30)
    so = _bubble_state(o[2], o[0])
    sp = to_cuda(to_cpu(_bubble_state(o[2], o[0])), torch.float32)
    ident = lambda s, f: s
    so = os_.step(so, 0.0, None, ident)
    sp = ps_.step(sp, 0.0, None, ident)
    for k in ("u", "v", "w"):
        assert rel_l2(sp[k], so[k]) < 1e-4, (k, rel_l2(sp[k], so[k]))
    # compare the carried perturbation (the float32 full field th_v cannot resolve it to 1e-4)
    th_p = sp["_sisl_state"][0].t["th_p"]
    assert rel_l2(th_p, so["th_v"] - o[2].theta_bg) < 1e-4


def test_ffsl_matches_oracle_and_conserves(mountain_pair):
    from oracle.steppers import FluxFormAdvector as OF
    from suetes_b200 import FluxFormAdvector as PF
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    gen = torch.Generator().manual_seed(3)
    rho = 1.0 + 0.1 * torch.rand(NX, NY, NZ, generator=gen, dtype=torch.float64)
    st = {"u": 15.0 * torch.ones(NX + 1, NY, NZ, dtype=torch.float64),
          "v": 5.0 * torch.ones(NX, NY + 1, NZ, dtype=torch.float64),
          "eta_dot": 1e-3 * torch.rand(NX, NY, NZ + 1, generator=gen, dtype=torch.float64)}
    st["u"][0] = 0.0
    st["u"][-1] = 0.0
    st["v"][:, 0] = 0.0
    st["v"][:, -1] = 0.0
    st["eta_dot"][:, :, 0] = 0.0
    st["eta_dot"][:, :, -1] = 0.0
    ref = OF(og, 100.0).advect_3d_split(rho, st, _bg(oph))
    out = PF(pg, 100.0, physics=pph).advect_3d_split(rho.cuda(), to_cuda(st), _bg(pph))
    assert rel_l2(out, ref) < 1e-12
    vol = (og.dx * og.dy / og.m_factors["m"][..., None] ** 2) * og.dz_m_full
    m0 = float((rho * vol).sum())
    m1 = float((out.double().cpu() * vol).sum())
    assert abs(m1 - m0) / m0 < 1e-14


def test_ffsl_1d_periodic_shift():
    """tests/test_periodic_boundaries.py:51-68 on the CUDA line kernel."""
    from suetes_b200 import FluxFormAdvector, RegionalGrid3D
    g = RegionalGrid3D(8, 4, 2, 1.0, 1.0, 1.0, 0.0, 0.0, device="cuda")
    adv = FluxFormAdvector(g, dt=1.0, periodic_axes=(0,))
    s = torch.tensor([1.0, 2.0, 4.0, 8.0, 16.0, 32.0, 64.0, 128.0], dtype=torch.float64, device="cuda")
    c = torch.ones(9, dtype=torch.float64, device="cuda")
    assert torch.allclose(adv.advect_1d(s, c, periodic=True), torch.roll(s, 1))
    assert torch.allclose(adv.advect_1d(s, -c, periodic=True), torch.roll(s, -1))


def test_gmres_float32_refinement_reaches_float64_accuracy(mountain_pair):
    """float32 GMRES with float64 iterative refinement converges to a
    tolerance the float32 residual cannot resolve (manufactured solution as
    tests/test_dynamical_core_3d.py:230-280) in as many cycles as float64."""
    from suetes_b200 import SemiImplicitSolver3D
    (og, oop, oph), (pg, pop, pph) = mountain_pair
    gen = torch.Generator().manual_seed(42)
    sh = shapes5(NX, NY, NZ)
    known = {k: torch.rand(sh[k], generator=gen, dtype=torch.float64) * s
             for k, s in (("u", 0.1), ("v", 0.1), ("w", 0.01), ("pi", 0.001), ("eta_dot", 0.001))}
    for k in ("w", "eta_dot"):
        known[k][:, :, 0] = 0.0
        known[k][:, :, -1] = 0.0
    bg = _bg(pph)
    rhs = pph.linear_operator(to_cuda(known), bg, dt=100.0, alpha=0.55)
    kw = dict(solver_tol=1e-9, solver_maxiter=40, solver_restart=100)
    s64 = SemiImplicitSolver3D(pph, 100.0, **kw)
    ref = s64.solve(rhs, bg)
    r32 = {k: v.float() for k, v in rhs.items()}
    s32 = SemiImplicitSolver3D(pph, 100.0, **kw)
    out = s32.solve(r32, bg)
    assert s32.last_info["converged"], s32.last_info
    assert s32.last_info["cycles"] <= s64.last_info["cycles"] + 1
    for k in ref:  # float32 rounding of the rhs, amplified by the conditioning
        assert rel_l2(out[k], ref[k]) < 1e-4, (k, rel_l2(out[k], ref[k]))
    plain = SemiImplicitSolver3D(pph, 100.0, refine=False, **kw)
    plain.solve(r32, bg)
    assert not plain.last_info["converged"]


@pytest.mark.parametrize("periodic", [(), (0,), (0, 1)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_metric_curvature_tendencies(periodic, dtype):
    """Euler3D.metric_curvature_tendencies (euler.py:188-206) on a 1500 km
    box at 60N, where the map-factor gradients are large."""
    kw = dict(lat=60.0, lon=30.0, h=mountain, periodic=periodic, dt=60.0)
    o = build("oracle", 16, 12, 6, 100000.0, 100000.0, 1000.0, **kw)
    p = build("cuda", 16, 12, 6, 100000.0, 100000.0, 1000.0, device="cuda", **kw)
    x = random_fields({"u": (17, 12, 6), "v": (16, 13, 6)}, 21, {"u": 20.0, "v": 20.0})
    ru, rv = o[2].metric_curvature_tendencies(x["u"], x["v"])
    pu, pv = p[2].metric_curvature_tendencies(x["u"].to("cuda", dtype), x["v"].to("cuda", dtype))
    assert float(ru.abs().max()) > 0.0 and float(rv.abs().max()) > 0.0
    assert rel_l2(pu, ru) < TOL[dtype], rel_l2(pu, ru)
    assert rel_l2(pv, rv) < TOL[dtype], rel_l2(pv, rv)
