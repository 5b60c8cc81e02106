"""The SISL step with a physics suite: CUDA path against the float64 oracle.

A toy suite with every hook the reference's ``PhysicsSuite`` offers
(suetes/physics/base.py): tendency schemes on u, v, w and th_v, an ML-style
closure fed ``ml_params``, an interior mask, a registered tracer carried by
the flux-form transport, and an update scheme that clips the tracer and
adjusts th_v.  Float64 agrees with the oracle to the GMRES tolerance (rel L2
<= 1e-8), float32 to 1e-4.
"""

import math

import pytest
import torch

from _cases import C, build, mountain, rel_l2, to_cpu, to_cuda

pytestmark = pytest.mark.gpu

NX, NY, NZ, DX, DZ, DT = 14, 12, 10, 500.0, 500.0, 10.0
KW = dict(dt=DT, N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1, damp_height=4000.0, max_damp=0.5)
SKW = dict(alpha=0.55, solver_tol=1e-12, solver_maxiter=60, solver_restart=30)


class Drag:
    def get_tendencies(self, state, bg):
        return {"u": -2e-3 * state["u"], "v": -2e-3 * state["v"], "w": -5e-3 * state["w"]}


class Newtonian:
    def get_tendencies(self, state, bg):
        return {"th_v": -(state["th_v"] - bg["th_v"]) / 600.0, "q": torch.zeros_like(state["th_v"])}


class Closure:
    is_ml_closure = True

    def get_tendencies(self, state, bg, ml_params=None):
        return {"u": ml_params["k"] * state["th_v_prime_u"]}


class ClipTracer:
    def apply_update(self, state):
        q = state["q"]
        return {"q": torch.clamp(q, min=0.0), "th_v": state["th_v"] + 5.0 * torch.clamp(-q, min=0.0)}


def _suite():
    from suetes_b200 import PhysicsSuite
    s = PhysicsSuite()
    for sch in (Drag(), Newtonian(), Closure()):
        s.add_tendency_scheme(sch)
    s.add_update_scheme(ClipTracer())
    s.register_tracer("q")
    return s


def _mask(device):
    i = torch.arange(NX + 1, dtype=torch.float64, device=device)
    mu = torch.clamp(torch.minimum(i, NX - i) / 3.0, max=1.0)[:, None, None]
    mm = 0.5 * (mu[1:] + mu[:-1])
    return {"u": mu, "th_v": mm}


def _state(ph, g):
    th = ph.theta_bg
    x, y, z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    r = torch.sqrt(x ** 2 + y ** 2 + (z - 1500.0) ** 2)
    blob = torch.where(r < 1000.0, torch.cos(0.5 * math.pi * r / 1000.0) ** 2, torch.zeros_like(r))
    th = th + 2.0 * blob
    rho = C["p0"] / (C["Rd"] * th) * ph.pi_bg ** (C["cvd"] / C["Rd"])
    z3 = lambda *s: torch.zeros(*s, dtype=torch.float64, device=th.device)
    return {"u": z3(NX + 1, NY, NZ) + 3.0, "v": z3(NX, NY + 1, NZ) - 2.0, "w": z3(NX, NY, NZ + 1),
            "eta_dot": z3(NX, NY, NZ + 1), "pi": ph.pi_bg.clone(), "th_v": th, "rho": rho,
            "q": 1e-3 * (blob - 0.05)}


def _pair(bc=None):
    from oracle.steppers import build_dynamical_core as obuild
    from suetes_b200 import build_dynamical_core as pbuild
    o = build("oracle", NX, NY, NZ, DX, DX, DZ, h=mountain, **KW)
    s0 = _state(o[2], o[0])
    ost, _ = obuild("sisl", o[0], o[1], C, dict(s0), physics_suite=_suite(), interior_mask=_mask("cpu"),
                    **KW, **SKW)
    p = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, device="cuda", **KW)
    pst, _ = pbuild("sisl", p[0], p[1], C, to_cuda(s0), physics_suite=_suite(), interior_mask=_mask("cuda"),
                    **KW, **SKW)
    return ost, pst, s0


ML = {"k": 0.01}
KEYS = ("u", "v", "w", "eta_dot", "rho", "q", "u_prev", "eta_dot_prev", "tend_th_v_prev", "tend_q_prev")


def _compare(sp, so, ph, tol):
    for k in KEYS:
        assert rel_l2(sp[k], so[k]) < tol, (k, rel_l2(sp[k], so[k]))
    for k, bg in (("pi", ph.pi_bg), ("th_v", ph.theta_bg)):
        assert rel_l2(sp[k].double().cpu() - bg, so[k] - bg) < tol, (k, rel_l2(sp[k].double().cpu() - bg, so[k] - bg))


def test_physics_suite_steps_match_oracle():
    ost, pst, s0 = _pair()
    so, sp = dict(s0), to_cuda(s0)
    ident = lambda s, f: s
    for n in range(2):
        so = ost.step(so, n * DT, None, ident, ml_params=ML)
        sp = pst.step(sp, n * DT, None, ident, ml_params=ML)
    _compare(sp, so, ost.physics, 1e-8)
    assert float(sp["q"].min()) >= 0.0


def test_physics_suite_with_lateral_relaxation():
    """The relaxation runs after the suite's state updates (steppers.py:1036-1040)."""
    from suetes_b200 import x_relaxation
    ost, pst, s0 = _pair()
    relax = x_relaxation(pst.physics.grid, 1500.0, 3.0)
    mm, mu, mv = (relax.mask_m.double().cpu(), relax.mask_u.double().cpu(), relax.mask_v.double().cpu())
    ph = ost.physics

    def obc(s, f):
        s = dict(s)
        for k, m, ext, bg in (("u", mu, 3.0, 0.0), ("v", mv, 0.0, 0.0), ("th_v", mm, 0.0, ph.theta_bg),
                              ("pi", mm, 0.0, ph.pi_bg)):
            s[k] = (1.0 - m[..., None]) * (s[k] - bg) + m[..., None] * ext + bg
        return s

    so = ost.step(dict(s0), 0.0, None, obc, ml_params=ML)
    sp = pst.step(to_cuda(s0), 0.0, None, relax, ml_params=ML)
    _compare(sp, so, ph, 1e-8)


def test_physics_suite_float32():
    ost, pst, s0 = _pair()
    ident = lambda s, f: s
    so = ost.step(dict(s0), 0.0, None, ident, ml_params=ML)
    pst.implicit_solver.solver_tol = 1e-6
    sp = pst.step(to_cuda(s0, torch.float32), 0.0, None, ident, ml_params=ML)
    for k in ("u", "v", "w", "q"):
        assert rel_l2(sp[k], so[k]) < 1e-4, (k, rel_l2(sp[k], so[k]))


def test_empty_suite_equals_plain_step():
    """No schemes: the physics path gives the plain step's fields bitwise
    (density to rounding: it is re-diagnosed from the assembled state)."""
    from suetes_b200 import PhysicsSuite, SISLStepper3D
    p = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, device="cuda", **KW)
    pe = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, device="cuda", physics_suite=PhysicsSuite(), **KW)
    s0 = to_cuda(to_cpu(_state(p[2], p[0])))
    s0.pop("q")
    ident = lambda s, f: s
    a = SISLStepper3D(p[2], DT, **SKW).step(dict(s0), 0.0, None, ident)
    b = SISLStepper3D(pe[2], DT, **SKW).step(dict(s0), 0.0, None, ident)
    for k in ("u", "v", "w", "eta_dot", "pi", "th_v", "tend_th_v_prev"):
        assert torch.equal(a[k], b[k]), k
    assert rel_l2(b["rho"], a["rho"]) < 1e-14


class PassiveTracer:
    """A suite that only registers a tracer (duck-typed, no PhysicsSuite)."""
    tracer_keys = ["q_test"]

    def get_explicit_tendencies(self, state, bg, interior_mask=None, ml_params=None):
        return {}

    def apply_state_updates(self, state):
        return state


def test_step_conserves_density_and_passive_tracer_mass():
    """Closed-box budgets through the final EOS and tracer reconciliation
    (the reference's tests/test_core_formula_regressions.py:238-292 case:
    8x8x5 flat box, dt 0.02, sinusoidal winds that vanish on the walls)."""
    from suetes_b200 import CGridOperator3D, Euler3D, RegionalGrid3D, SISLStepper3D
    dt = 0.02
    flat = lambda x, y: 0.0 * (x + y)
    g = RegionalGrid3D(8, 8, 5, 2000.0, 2000.0, 500.0, 45.0, 0.0, h_func=flat, device="cuda")
    op = CGridOperator3D(g)
    ph = Euler3D(g, op, C, dt=dt, N_bv=0.0, damp_height=1e9, max_damp=0.0, nu_div_factor=0.0, nu_h_factor=0.0,
                 physics_suite=PassiveTracer())
    c = C
    f64 = dict(dtype=torch.float64, device="cuda")
    rho = c["p0"] / (c["Rd"] * ph.theta_bg) * ph.pi_bg ** (c["cvd"] / c["Rd"])
    i_u = torch.arange(9, **f64)[:, None, None]
    j_v = torch.arange(9, **f64)[None, :, None]
    x = torch.arange(8, **f64)[:, None, None]
    y = torch.arange(8, **f64)[None, :, None]
    state = {"u": 2.0 * torch.sin(math.pi * i_u / 8) + torch.zeros(9, 8, 5, **f64),
             "v": -1.5 * torch.sin(math.pi * j_v / 8) + torch.zeros(8, 9, 5, **f64),
             "w": torch.zeros(8, 8, 6, **f64), "eta_dot": torch.zeros(8, 8, 6, **f64),
             "pi": ph.pi_bg.clone(), "th_v": ph.theta_bg.clone(), "rho": rho,
             "q_test": 1.0 + 0.2 * torch.sin(2 * math.pi * x / 8) * torch.cos(2 * math.pi * y / 8)
             + torch.zeros(8, 8, 5, **f64)}
    vol = g.dx * g.dy * g.dz_m_full / g.m_factors["m"][..., None] ** 2
    mass0 = float((state["rho"] * vol).sum())
    tracer0 = float((state["rho"] * state["q_test"] * vol).sum())
    st = SISLStepper3D(ph, dt, alpha=0.5, solver_tol=1e-11, solver_maxiter=80, solver_restart=40)
    bg = ph.precompute_bg(ph.bg_state_ref())
    moved = st.ffsl_advector.advect_3d_split(state["rho"] * state["q_test"], state, bg)
    res = st.step(state, 0.0, None, lambda s, f: s)
    mass1 = float((res["rho"] * vol).sum())
    tracer1 = float((res["rho"] * res["q_test"] * vol).sum())
    assert abs(mass1 - mass0) / mass0 < 1e-10
    assert abs(tracer1 - tracer0) / tracer0 < 1e-10
    assert rel_l2(res["rho"] * res["q_test"], moved) < 1e-12
