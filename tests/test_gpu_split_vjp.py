"""Native reverse sweep of the split-explicit RK3 core (sisl_split_step_vjp)
against the float64 oracle's autograd of the same three stages.

The map is SplitExplicitStepper3D.step's stage loop (steppers.py:1117-1231:
slow tendencies with the step start's hyperdiffusion, 3rd-order upwind
advection, the acoustic sub-cycles with the vertically implicit column
solve, the eta_dot diagnosis between stages) from a diagnosed state;
autograd of the oracle carries the reference's stop_gradient on padded
stagger copies and no cotangent through jnp.sign of the upwind flux.
Float64 agrees to rounding, float32 to its precision; the fixed-point
scatters make the sweep bitwise repeatable.
"""

import pytest
import torch

from _cases import build, mountain, rel_l2
from test_gpu_split import DX, DZ, KW, NX, NY, NZ, _state

pytestmark = pytest.mark.gpu

IN = ("u", "v", "w", "eta_dot", "pi", "th_v")
NATIVE = {"u": "u", "v": "v", "w": "w", "eta_dot": "eta_dot", "pi": "pi_p", "th_v": "th_p"}


def _oracle_stages(ost, st):
    """The oracle step's stages (oracle/split_explicit.py step) from a diagnosed state."""
    ph = ost.physics
    bg = ost._bg()
    sp, _ = ost._prime(st)
    diff = ph.diffusion.get_tendencies(sp, bg_precomputed=bg) if (ph.nu_h > 0.0 or ph.nu_div > 0.0) else {}
    nu_h = ph.nu_h
    ph.nu_h = 0.0
    try:
        cur = st
        stages = ((ost.dtau_stage1, ost.ns_stage1), (ost.dtau_stage2, ost.ns_stage2),
                  (ost.dtau_stage3, ost.ns_stage3))
        for n, (dtau, ns) in enumerate(stages):
            sf = ost._compute_slow_tendencies(cur, bg, {}, diff, None)
            cur = ost._acoustic_loop(st, cur, sf, bg, dtau, ns)
            if n < 2:
                cur = dict(cur)
                cur["eta_dot"], cur["w"] = ost._diagnose_eta_dot(cur)
    finally:
        ph.nu_h = nu_h
    return cur


def _setup(periodic, ns=4, dt=2.0, **kw):
    from oracle.split_explicit import SplitExplicitStepper3D as OSp
    from suetes_b200 import SplitExplicitStepper3D as PSp
    ekw = dict(KW, **kw)
    o = build("oracle", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=periodic, dt=dt, **ekw)
    p = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=periodic, device="cuda", dt=dt, **ekw)
    ost, pst = OSp(o[2], dt, ns, alpha=0.5), PSp(p[2], dt, ns, alpha=0.5)
    s0 = _state(o[2], o[0])
    s0.pop("q")
    s0["eta_dot"], s0["w"] = ost._diagnose_eta_dot(s0)
    return ost, pst, s0


def _oracle_vjp(ost, s0, cot):
    leaves = {k: s0[k].clone().requires_grad_(True) for k in IN}
    st = dict(s0, **leaves)
    out = _oracle_stages(ost, st)
    J = sum((out[k] * cot[k]).sum() for k in IN)
    g = torch.autograd.grad(J, [leaves[k] for k in IN], allow_unused=True)
    return {k: (gk if gk is not None else torch.zeros_like(s0[k])) for k, gk in zip(IN, g)}


def _native_vjp(pst, s0, cot, dtype, deterministic=True):
    ph = pst.physics
    core = pst.core(dtype)
    f = core.field

    def cu(t):
        return t.detach().to("cuda", torch.float64)

    st = {"u": f(cu(s0["u"]), "u"), "v": f(cu(s0["v"]), "v"), "w": f(cu(s0["w"]), "w"),
          "eta_dot": f(cu(s0["eta_dot"]), "w"),
          "pi_p": f(cu(s0["pi"]) - ph.pi_bg, "m"), "th_p": f(cu(s0["th_v"]) - ph.theta_bg, "m"),
          "rho": f(cu(s0["rho"]), "m")}
    locs = {"u": "u", "v": "v", "w": "w", "eta_dot": "w", "pi": "m", "th_v": "m"}
    ob = {NATIVE[k]: f(cu(cot[k]), locs[k]) for k in IN}
    return pst.step_vjp_device(core, st, ob, deterministic=deterministic)


def _cotangents(s0, seed=3):
    gen = torch.Generator().manual_seed(seed)
    return {k: torch.randn(tuple(s0[k].shape), generator=gen, dtype=torch.float64) for k in IN}


@pytest.mark.parametrize("periodic", [(), (0,), (0, 1)])
def test_split_vjp_matches_oracle_autograd(periodic):
    ost, pst, s0 = _setup(periodic)
    cot = _cotangents(s0)
    ref = _oracle_vjp(ost, s0, cot)
    for det in (True, False):  # fixed-point and float atomic scatters
        got = _native_vjp(pst, s0, cot, torch.float64, deterministic=det)
        errs = {k: rel_l2(got[NATIVE[k]], ref[k]) for k in IN}
        assert max(errs.values()) < 1e-9, (periodic, det, errs)
    assert float(ref["th_v"].abs().max()) > 0.0


def test_split_vjp_without_divergence_damping_and_float32():
    """nu_div = 0 (no stage hyperdiffusion, no damping gradient) in float64,
    and the default configuration in float32 against the float64 oracle."""
    ost, pst, s0 = _setup((), nu_div_factor=0.0)
    cot = _cotangents(s0, 5)
    ref = _oracle_vjp(ost, s0, cot)
    got = _native_vjp(pst, s0, cot, torch.float64)
    errs = {k: rel_l2(got[NATIVE[k]], ref[k]) for k in IN}
    assert max(errs.values()) < 1e-9, errs
    ost, pst, s0 = _setup(())
    cot = _cotangents(s0, 7)
    ref = _oracle_vjp(ost, s0, cot)
    got = _native_vjp(pst, s0, cot, torch.float32)
    errs = {k: rel_l2(got[NATIVE[k]].double(), ref[k]) for k in IN}
    assert max(errs.values()) < 1e-4, errs


def test_split_vjp_is_bitwise_repeatable():
    ost, pst, s0 = _setup((0,))
    cot = _cotangents(s0, 9)
    runs = [_native_vjp(pst, s0, cot, torch.float32) for _ in range(3)]
    for r in runs[1:]:
        for k in NATIVE.values():
            assert torch.equal(r[k], runs[0][k]), k


def _bc_mix(s, forcing):
    """An elementwise bc_fn that couples fields (same on both sides)."""
    out = dict(s)
    out["u"] = 0.9 * s["u"]
    out["th_v"] = s["th_v"] + 0.05 * (s["pi"] - 1.0)
    return out


@pytest.mark.parametrize("bc", [None, _bc_mix])
def test_split_step_vjp_matches_oracle_autograd(bc):
    """The whole step (input diagnosis, the stages, bc_fn, the final
    diagnosis and the equation of state) against autograd of the oracle's
    SplitExplicitStepper3D.step, float64, periodic in x."""
    from oracle.split_explicit import SplitExplicitStepper3D as OSp
    from suetes_b200 import SplitExplicitStepper3D as PSp
    o = build("oracle", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=(0,), dt=2.0, **KW)
    p = build("cuda", NX, NY, NZ, DX, DX, DZ, h=mountain, periodic=(0,), device="cuda", dt=2.0, **KW)
    ost, pst = OSp(o[2], 2.0, 4, alpha=0.5), PSp(p[2], 2.0, 4, alpha=0.5)
    s = _state(o[2], o[0])
    s.pop("q")
    keys = ("u", "v", "w", "eta_dot", "pi", "th_v", "rho")
    gen = torch.Generator().manual_seed(13)
    cot = {k: torch.randn(tuple(s[k].shape), generator=gen, dtype=torch.float64) for k in keys}
    leaves = {k: s[k].clone().requires_grad_(True) for k in ("u", "v", "w", "pi", "th_v", "rho")}
    ident = (lambda a, f: a) if bc is None else bc
    out_o = ost.step(dict(s, **leaves), 0.0, None, ident)
    J = sum((out_o[k] * cot[k]).sum() for k in keys)
    ref = dict(zip(leaves, torch.autograd.grad(J, list(leaves.values()), allow_unused=True)))
    sc = {k: (v.to("cuda") if torch.is_tensor(v) else v) for k, v in s.items()}
    out_p, got = pst.step_vjp(sc, {k: v.to("cuda") for k, v in cot.items()}, bc_fn=bc)
    for k in ("u", "v", "w", "pi", "th_v"):
        assert rel_l2(out_p[k], out_o[k].detach()) < 1e-10, k
        e = rel_l2(got[k], ref[k])
        assert e < 1e-9, (k, e)
    assert float(got["rho"].abs().max()) == 0.0 and (ref["rho"] is None or float(ref["rho"].abs().max()) == 0.0)
    assert float(got["eta_dot"].abs().max()) == 0.0
