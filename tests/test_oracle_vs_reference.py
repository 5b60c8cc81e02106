"""The float64 oracle against the reference's own JAX core, where that can run.

The build image has no JAX, so every test here skips unless ``import jax``
works and the environment variable ``SUETES_REFERENCE`` names a checkout of
the reference (the directory that holds its ``suetes`` package).  On such a
machine this pins the oracle -- and through the GPU parity tests the CUDA
kernels -- to the reference itself: the Helmholtz operator, one full SISL
step (steppers.py:720-1073) at a tight GMRES tolerance, and the gradient of
that step under ``jax.grad`` against the oracle's autograd.  GMRES iterates
are not compared (JAX's restart internals are not part of the contract).
CPU only; the GPU tests never read the reference.
"""

import os
import sys

import numpy as np
import pytest
import torch

from _cases import C

jax = pytest.importorskip("jax")
REF = os.environ.get("SUETES_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "suetes")):
    pytest.skip("SUETES_REFERENCE does not name a reference checkout", allow_module_level=True)
jax.config.update("jax_enable_x64", True)
import jax.numpy as jnp  # noqa: E402

if REF not in sys.path:
    sys.path.insert(0, REF)

NX, NY, NZ, DX, DZ, DT = 12, 10, 8, 500.0, 500.0, 10.0
KW = dict(N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1, damp_height=3000.0, max_damp=0.5)


def _hill(x, y):
    xp = torch if isinstance(x, torch.Tensor) else jnp
    return 300.0 * xp.exp(-(x ** 2 + y ** 2) / 2000.0 ** 2)


def _both():
    from suetes.regional3d.euler import Euler3D as RE
    from suetes.regional3d.geometry import RegionalGrid3D as RG
    from suetes.regional3d.operators import CGridOperator3D as RO
    from oracle.euler import Euler3D as OE
    from oracle.grid import RegionalGrid3D as OG
    from oracle.ops import CGridOperator3D as OO
    args = (NX, NY, NZ, DX, DX, DZ, 45.0, 0.0)
    og, rg = OG(*args, h_func=_hill), RG(*args, h_func=_hill)
    return (og, OO(og), OE(og, OO(og), C, dt=DT, **KW)), (rg, RO(rg), RE(rg, RO(rg), C, dt=DT, **KW))


def _np(t):
    return np.asarray(t.detach().cpu().numpy() if torch.is_tensor(t) else t, dtype=np.float64)


def _rel(a, b):
    a, b = _np(a), _np(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _state(oph, g):
    gen = torch.Generator().manual_seed(7)
    r = lambda *s: torch.randn(*s, generator=gen, dtype=torch.float64)
    w = 0.05 * r(NX, NY, NZ + 1)
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
    th = oph.theta_bg + 0.5 * r(NX, NY, NZ)
    rho = C["p0"] / (C["Rd"] * th) * oph.pi_bg ** (C["cvd"] / C["Rd"])
    return {"u": 5.0 + r(NX + 1, NY, NZ), "v": -2.0 + r(NX, NY + 1, NZ), "w": w,
            "eta_dot": torch.zeros(NX, NY, NZ + 1, dtype=torch.float64),
            "pi": oph.pi_bg + 1e-5 * r(NX, NY, NZ), "th_v": th, "rho": rho}


def test_background_and_operator_match_reference():
    (og, oo, oph), (rg, ro, rph) = _both()
    assert _rel(rph.theta_bg, oph.theta_bg) < 1e-13
    assert _rel(rph.pi_bg, oph.pi_bg) < 1e-13
    obg = oph.precompute_bg(oph.bg_state_ref())
    rbg = rph.precompute_bg({"rho": C["p0"] / (C["Rd"] * rph.theta_bg) * rph.pi_bg ** (C["cvd"] / C["Rd"]),
                             "pi": rph.pi_bg, "th_v": rph.theta_bg})
    for k in obg:
        assert _rel(rbg[k], obg[k]) < 1e-12, k
    gen = torch.Generator().manual_seed(3)
    x = {k: torch.randn(*s, generator=gen, dtype=torch.float64) * sc for k, s, sc in
         (("u", (NX + 1, NY, NZ), 0.1), ("v", (NX, NY + 1, NZ), 0.1), ("w", (NX, NY, NZ + 1), 0.01),
          ("pi", (NX, NY, NZ), 1e-3), ("eta_dot", (NX, NY, NZ + 1), 1e-3))}
    ref = rph.linear_operator({k: jnp.asarray(_np(v)) for k, v in x.items()}, rbg, DT, alpha=0.55)
    out = oph.linear_operator(x, obg, DT, alpha=0.55)
    for k in out:
        assert _rel(out[k], ref[k]) < 1e-12, k


def _steppers(oph, rph, s_np):
    from oracle.steppers import build_dynamical_core as obuild
    from suetes.regional3d.steppers import build_dynamical_core as rbuild
    skw = dict(dt=DT, solver_tol=1e-12, solver_maxiter=60, solver_restart=40, **KW)
    so = {k: torch.as_tensor(v) for k, v in s_np.items()}
    sr = {k: jnp.asarray(v) for k, v in s_np.items()}
    ost, _ = obuild("sisl", oph.grid, oph.op, C, so, **skw)
    rst, _ = rbuild("sisl", rph.grid, rph.op, C, sr, **skw)
    sr["is_first_step"] = jnp.asarray(1.0)
    return ost, so, rst, sr


def test_one_step_matches_reference():
    (og, oo, oph), (rg, ro, rph) = _both()
    s_np = {k: _np(v) for k, v in _state(oph, og).items()}
    ost, so, rst, sr = _steppers(oph, rph, s_np)
    ident = lambda s, f: s
    out_o = ost.step(so, 0.0, None, ident)
    out_r = rst.step(sr, 0.0, None, ident)
    for k in ("u", "v", "w", "eta_dot", "pi", "th_v", "rho"):
        assert _rel(out_o[k], out_r[k]) < 1e-8, (k, _rel(out_o[k], out_r[k]))


def test_step_gradient_matches_reference():
    (og, oo, oph), (rg, ro, rph) = _both()
    s_np = {k: _np(v) for k, v in _state(oph, og).items()}
    ost, so, rst, sr = _steppers(oph, rph, s_np)
    gen = np.random.default_rng(11)
    wt = gen.standard_normal(s_np["th_v"].shape)
    wu = gen.standard_normal(s_np["u"].shape)
    ident = lambda s, f: s

    def jfun(th):
        out = rst.step(dict(sr, th_v=th), 0.0, None, ident)
        return jnp.sum(jnp.asarray(wt) * out["th_v"]) + jnp.sum(jnp.asarray(wu) * out["u"])
    g_ref = jax.grad(jfun)(sr["th_v"])
    th = so["th_v"].clone().requires_grad_(True)
    out = ost.step(dict(so, th_v=th), 0.0, None, ident)
    J = (torch.as_tensor(wt) * out["th_v"]).sum() + (torch.as_tensor(wu) * out["u"]).sum()
    (g,) = torch.autograd.grad(J, th)
    assert _rel(g, g_ref) < 1e-7, _rel(g, g_ref)
