"""The split-explicit RK3 core on the GPU against the float64 oracle.

``SplitExplicitStepper3D.step`` (steppers.py:1117-1270) through
``sisl_split_step``: three RK3 stages of slow tendencies (explicit dynamics,
3rd-order upwind flux advection, hyperdiffusion of the step start and --
with divergence damping on -- of the stage) and acoustic sub-cycles with the
vertically implicit column solve.  Float64 agrees with the oracle to
rounding over two steps (rel L2 <= 1e-10), float32 within 5e-5 after one
step (w 2.8e-5, the winds ~1e-6: w is the small residual of the
acoustic balance); the closed-box
budgets of the reference's tests/test_core_formula_regressions.py:238-292
hold through the GPU path.
"""

import math

import pytest
import torch

from _cases import C, build, mountain, rel_l2, to_cuda

pytestmark = pytest.mark.gpu

NX, NY, NZ, DX, DZ = 14, 12, 10, 500.0, 500.0
KW = dict(N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1, damp_height=3000.0, max_damp=0.5)


def _state(ph, g, u0=3.0, v0=-2.0):
    th = ph.theta_bg
    x, y, z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    r = torch.sqrt(x ** 2 + y ** 2 + (z - 1500.0) ** 2)
    blob = torch.where(r < 1000.0, torch.cos(0.5 * math.pi * r / 1000.0) ** 2, torch.zeros_like(r))
    th = th + 2.0 * blob
    rho = C["p0"] / (C["Rd"] * th) * ph.pi_bg ** (C["cvd"] / C["Rd"])
    z3 = lambda *s: torch.zeros(*s, dtype=torch.float64, device=th.device)
    gen = torch.Generator(device=th.device).manual_seed(5)
    w = 0.05 * torch.randn(NX, NY, NZ + 1, dtype=torch.float64, device=th.device, generator=gen)
    return {"u": z3(NX + 1, NY, NZ) + u0, "v": z3(NX, NY + 1, NZ) + v0, "w": w,
            "eta_dot": z3(NX, NY, NZ + 1), "pi": ph.pi_bg.clone(), "th_v": th, "rho": rho,
            "q": 1e-3 * (blob + 0.1)}


def _pair(dt, ns, periodic=(), suite=None, **kw):
    from oracle.split_explicit import SplitExplicitStepper3D as OSp
    from suetes_b200 import SplitExplicitStepper3D as PSp
    ekw = dict(KW, **kw)
    o = build("oracle", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=periodic, dt=dt, physics_suite=suite, **ekw)
    p = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=periodic, device="cuda", dt=dt,
              physics_suite=suite, **ekw)
    return OSp(o[2], dt, ns, alpha=0.5), PSp(p[2], dt, ns, alpha=0.5), o


def _compare(sp, so, ph, tol, keys=("u", "v", "w", "eta_dot", "rho")):
    for k in keys:
        assert rel_l2(sp[k], so[k]) < tol, (k, rel_l2(sp[k], so[k]))
    for k, bg in (("pi", ph.pi_bg), ("th_v", ph.theta_bg)):
        e = rel_l2(sp[k].double().cpu() - bg, so[k] - bg)
        assert e < tol, (k, e)


@pytest.mark.parametrize("periodic", [(), (0,), (0, 1)])
def test_split_steps_match_oracle(periodic):
    ost, pst, o = _pair(2.0, 4, periodic)
    s0 = _state(o[2], o[0])
    s0.pop("q")
    so, sp = dict(s0), to_cuda(s0)
    ident = lambda s, f: s
    for n in range(2):
        so = ost.step(so, n * 2.0, None, ident)
        sp = pst.step(sp, n * 2.0, None, ident)
    _compare(sp, so, o[2], 1e-10)
    # the acoustic cycle moved the fields: not a trivial pass-through
    assert rel_l2(sp["w"], to_cuda(s0)["w"]) > 1e-3


@pytest.mark.parametrize("ns", [1, 3, 6])
def test_split_stage_counts(ns):
    """round(ns/3), round(ns/2), ns acoustic steps per stage (banker's rounding)."""
    ost, pst, o = _pair(1.5, ns, nu_div_factor=0.0)
    assert (pst.ns_stage1, pst.ns_stage2, pst.ns_stage3) == (ost.ns_stage1, ost.ns_stage2, ost.ns_stage3)
    s0 = _state(o[2], o[0])
    s0.pop("q")
    so = ost.step(dict(s0), 0.0, None, lambda s, f: s)
    sp = pst.step(to_cuda(s0), 0.0, None, lambda s, f: s)
    _compare(sp, so, o[2], 1e-10)


class _Suite:
    """Drag, Newtonian relaxation and a passive tracer (duck-typed suite)."""
    tracer_keys = ["q"]

    def get_explicit_tendencies(self, state, bg, interior_mask=None, ml_params=None):
        return {"u": -2e-3 * state["u"], "w": -5e-3 * state["w"], "th_v": -(state["th_v"] - bg["th_v"]) / 600.0}

    def apply_state_updates(self, state):
        out = dict(state)
        out["q"] = torch.clamp(state["q"], min=0.0)
        return out


def test_split_with_physics_suite_and_tracer():
    ost, pst, o = _pair(2.0, 4, suite=_Suite())
    s0 = _state(o[2], o[0])
    so = ost.step(dict(s0), 0.0, None, lambda s, f: s)
    sp = pst.step(to_cuda(s0), 0.0, None, lambda s, f: s)
    _compare(sp, so, o[2], 1e-10, keys=("u", "v", "w", "eta_dot", "rho", "q"))


def test_split_float32_close_to_float64():
    ost, pst, o = _pair(2.0, 4)
    s0 = _state(o[2], o[0])
    s0.pop("q")
    so = ost.step(dict(s0), 0.0, None, lambda s, f: s)
    sp = pst.step(to_cuda(s0, torch.float32), 0.0, None, lambda s, f: s)
    for k in ("u", "v", "w"):
        assert rel_l2(sp[k], so[k]) < 5e-5, (k, rel_l2(sp[k], so[k]))


class _PassiveTracer:
    tracer_keys = ["q_test"]

    def get_explicit_tendencies(self, state, bg, interior_mask=None, ml_params=None):
        return {}

    def apply_state_updates(self, state):
        return state


def test_split_conserves_density_and_passive_tracer_mass():
    """tests/test_core_formula_regressions.py:238-292, split_explicit case."""
    from suetes_b200 import CGridOperator3D, Euler3D, RegionalGrid3D, SplitExplicitStepper3D
    dt = 0.02
    g = RegionalGrid3D(8, 8, 5, 2000.0, 2000.0, 500.0, 45.0, 0.0, h_func=lambda x, y: 0.0 * (x + y), device="cuda")
    ph = Euler3D(g, CGridOperator3D(g), C, dt=dt, N_bv=0.0, damp_height=1e9, max_damp=0.0, nu_div_factor=0.0,
                 nu_h_factor=0.0, physics_suite=_PassiveTracer())
    f64 = dict(dtype=torch.float64, device="cuda")
    rho = C["p0"] / (C["Rd"] * ph.theta_bg) * ph.pi_bg ** (C["cvd"] / C["Rd"])
    iu = torch.arange(9, **f64)[:, None, None]
    jv = torch.arange(9, **f64)[None, :, None]
    x = torch.arange(8, **f64)[:, None, None]
    y = torch.arange(8, **f64)[None, :, None]
    state = {"u": 2.0 * torch.sin(math.pi * iu / 8) + torch.zeros(9, 8, 5, **f64),
             "v": -1.5 * torch.sin(math.pi * jv / 8) + torch.zeros(8, 9, 5, **f64),
             "w": torch.zeros(8, 8, 6, **f64), "eta_dot": torch.zeros(8, 8, 6, **f64),
             "pi": ph.pi_bg.clone(), "th_v": ph.theta_bg.clone(), "rho": rho,
             "q_test": 1.0 + 0.2 * torch.sin(2 * math.pi * x / 8) * torch.cos(2 * math.pi * y / 8)
             + torch.zeros(8, 8, 5, **f64)}
    vol = g.dx * g.dy * g.dz_m_full / g.m_factors["m"][..., None] ** 2
    mass0 = float((state["rho"] * vol).sum())
    tracer0 = float((state["rho"] * state["q_test"] * vol).sum())
    st = SplitExplicitStepper3D(ph, dt, ns=2, alpha=0.5)
    bg = ph.precompute_bg(ph.bg_state_ref())
    moved = st.ffsl_advector.advect_3d_split(state["rho"] * state["q_test"], state, bg)
    res = st.step(state, 0.0, None, lambda s, f: s)
    assert abs(float((res["rho"] * vol).sum()) - mass0) / mass0 < 1e-10
    assert abs(float((res["rho"] * res["q_test"] * vol).sum()) - tracer0) / tracer0 < 1e-10
    assert rel_l2(res["rho"] * res["q_test"], moved) < 1e-12


def test_split_with_lateral_relaxation():
    """bc_fn after the stages (steppers.py:1249-1253): the LateralRelaxation
    blend against the same blend written out for the oracle."""
    from suetes_b200 import x_relaxation
    ost, pst, o = _pair(2.0, 4)
    ph = o[2]
    relax = x_relaxation(pst.physics.grid, 1500.0, 3.0)
    mm, mu, mv = (relax.mask_m.double().cpu(), relax.mask_u.double().cpu(), relax.mask_v.double().cpu())

    def obc(s, f):
        s = dict(s)
        for k, m, ext, bg in (("u", mu, 3.0, 0.0), ("v", mv, 0.0, 0.0), ("th_v", mm, 0.0, ph.theta_bg),
                              ("pi", mm, 0.0, ph.pi_bg)):
            s[k] = (1.0 - m[..., None]) * (s[k] - bg) + m[..., None] * ext + bg
        return s

    s0 = _state(o[2], o[0])
    s0.pop("q")
    so = ost.step(dict(s0), 0.0, None, obc)
    sp = pst.step(to_cuda(s0), 0.0, None, relax)
    _compare(sp, so, ph, 1e-10)
