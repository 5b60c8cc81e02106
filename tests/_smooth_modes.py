"""Smooth-mode timestep refinement (verification/smooth_mode_core_convergence.py),
shared by the oracle test (CPU) and the CUDA test.

A small-amplitude standing buoyancy mode ("gravity") and a standing acoustic
mode ("acoustic") on a 32 x 3 x 16 Cartesian channel (map factors one, no
Coriolis, no damping or diffusion), integrated with a timestep-halving family
on one fixed grid.  Errors are differences between successive refinements
(lateral boundary stencils cropped), and the order is log2 of the ratio of
successive errors; the reference gates the finest order at 1.7 for both
cores (:210-218, :246-252)."""

import math

import torch

C = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}
LX, LY, LZ = 20_000.0, 1_875.0, 10_000.0
CASES = {  # smooth_mode_core_convergence.py:64-71
    "gravity": {"t_end": 20.0, "dt": [2.0, 1.0, 0.5, 0.25], "fields": ("th_v", "w")},
    "acoustic": {"t_end": 10.0, "dt": [1.0, 0.5, 0.25, 0.125], "fields": ("pi", "u")},
}
WAVE_ORDER = 1.7


def _modules(pkg):
    if pkg == "oracle":
        from oracle.grid import RegionalGrid3D
        from oracle.ops import CGridOperator3D
        from oracle.euler import Euler3D
        from oracle.steppers import build_dynamical_core
    else:
        from suetes_b200 import RegionalGrid3D, CGridOperator3D, Euler3D, build_dynamical_core
    return RegionalGrid3D, CGridOperator3D, Euler3D, build_dynamical_core


def _grid(pkg, nx, nz, device):
    """The Cartesian channel of :74-84: unit map factors, no map-factor
    gradients, no Coriolis."""
    RegionalGrid3D = _modules(pkg)[0]
    kw = {} if pkg == "oracle" else {"device": device}
    g = RegionalGrid3D(nx, 3, nz, LX / nx, LY / 3, LZ / nz, 0.0, 0.0, **kw)
    for key in g.m_factors:
        g.m_factors[key] = torch.ones_like(g.m_factors[key])
    g.dm_dx_m = torch.zeros_like(g.dm_dx_m)
    g.dm_dy_m = torch.zeros_like(g.dm_dy_m)
    g.f_u = torch.zeros_like(g.f_u)
    g.f_v = torch.zeros_like(g.f_v)
    return g


def _initial_state(case, g, ph):
    """:87-127 (the tracer case is left out)."""
    z = lambda *s: torch.zeros(*s, dtype=torch.float64)
    nx, ny, nz = g.nx, g.ny, g.nz
    th, pi = ph.theta_bg.double().cpu(), ph.pi_bg.double().cpu()
    st = {"u": z(nx + 1, ny, nz), "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1), "eta_dot": z(nx, ny, nz + 1),
          "pi": pi.clone(), "th_v": th.clone()}
    x = g.x_m.double().cpu()[:, None, None]
    zz = g.z_m.double().cpu()[None, None, :]
    if case == "gravity":
        st["th_v"] = th + 1.0e-2 * (torch.cos(2.0 * math.pi * x / LX) * torch.sin(math.pi * zz / LZ))
    else:
        st["pi"] = pi + 1.0e-6 * torch.cos(2.0 * math.pi * x / LX) + 0.0 * zz
    st["rho"] = C["p0"] / (C["Rd"] * st["th_v"]) * st["pi"] ** (C["cvd"] / C["Rd"])
    return st


def run(pkg, case, core, dt, nx=32, nz=16, device=None):
    """Fields of CASES[case] after t_end (:130-174), float64 on the CPU."""
    RegionalGrid3D, CGridOperator3D, Euler3D, build = _modules(pkg)
    g = _grid(pkg, nx, nz, device)
    op = CGridOperator3D(g)
    nb = 0.01 if case == "gravity" else 0.0
    damp = dict(damp_height=1.0e9, max_damp=0.0, nu_h_factor=0.0, nu_div_factor=0.0)
    ph = Euler3D(g, op, C, dt=dt, N_bv=nb, **damp)
    st0 = _initial_state(case, g, ph)
    if pkg != "oracle":
        st0 = {k: v.to(device) for k, v in st0.items()}
    kw = dict(dt=dt, alpha=0.5, N_bv=nb, **damp)
    if core == "sisl":
        kw.update(solver_tol=1.0e-10, solver_maxiter=80, solver_restart=40)
    else:
        kw["ns"] = 12
    stepper, adt = build(core, g, op, C, st0, **kw)
    steps = round(CASES[case]["t_end"] / adt)
    st = st0
    bc = (lambda s, f: s) if pkg == "oracle" else None
    with torch.no_grad():
        for n in range(steps):
            st = stepper.step(st, n * adt, None, bc)
    return {f: st[f].detach().double().cpu() for f in CASES[case]["fields"]}


def _cropped(f):  # :177-183
    f = f[4:-4]
    return f[:, :, 2:-2] if f.shape[2] > 8 else f


def orders(solutions, fields):
    """Self-convergence errors and orders (:186-207)."""
    errs = {f: [] for f in fields}
    for a, b in zip(solutions[:-1], solutions[1:]):
        for f in fields:
            d = _cropped(a[f]) - _cropped(b[f])
            errs[f].append(float(torch.linalg.vector_norm(d) / max(float(torch.linalg.vector_norm(_cropped(b[f]))),
                                                                     1e-300)))
    rates = {f: [math.log2(x / y) for x, y in zip(v[:-1], v[1:])] for f, v in errs.items()}
    return errs, rates
