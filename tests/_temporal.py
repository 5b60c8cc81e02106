"""Pure temporal self-convergence (verification/temporal_core_convergence.py):
the 2 K warm bubble on a 40 x 3 x 40 Cartesian slab (dx = 250 m, no map
factors or Coriolis, no damping or diffusion, alpha 0.5; SISL GMRES tol
1e-12, split-explicit with a fixed ns = 40) integrated to t = 24 s with a
timestep-halving family; the fields are compared on the centre y row at
mass points, 1500 m in from the boundaries (:48-200)."""

import math

import torch

C = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}


def run(core, dt, dx=250.0, t_end=24.0):
    from oracle.grid import RegionalGrid3D
    from oracle.ops import CGridOperator3D
    from oracle.euler import Euler3D
    from oracle.steppers import build_dynamical_core
    nx = nz = int(10000 / dx)
    ny = 3
    g = RegionalGrid3D(nx, ny, nz, dx, dx, dx, 0.0, 0.0)
    for k in g.m_factors:
        g.m_factors[k] = torch.ones_like(g.m_factors[k])
    g.dm_dx_m, g.dm_dy_m = torch.zeros_like(g.dm_dx_m), torch.zeros_like(g.dm_dy_m)
    g.f_u, g.f_v = torch.zeros_like(g.f_u), torch.zeros_like(g.f_v)
    op = CGridOperator3D(g)
    tp = Euler3D(g, op, C, dt=dt)
    z = lambda *s: torch.zeros(*s, dtype=torch.float64)
    X, _, Z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    r = torch.sqrt(X ** 2 + (Z - 2000.0) ** 2)
    bubble = torch.where(r <= 1500.0, 2.0 * torch.cos(0.5 * math.pi * r / 1500.0) ** 2, torch.zeros_like(r))
    th = tp.theta_bg + bubble
    st = {"u": z(nx + 1, ny, nz), "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1), "pi": tp.pi_bg.clone(),
          "eta_dot": z(nx, ny, nz + 1), "th_v": th,
          "rho": C["p0"] / (C["Rd"] * th) * tp.pi_bg ** (C["cvd"] / C["Rd"])}
    st.update(u_prev=st["u"], v_prev=st["v"], w_prev=st["w"], eta_dot_prev=st["eta_dot"],
              tend_th_v_prev=z(nx, ny, nz), is_first_step=1.0)
    kw = dict(dt=dt, nu_div_factor=0.0, nu_h_factor=0.0, damp_height=7500.0, max_damp=0.0, alpha=0.5)
    if core == "sisl":
        kw.update(solver_tol=1e-12, solver_maxiter=20, solver_restart=20)
    else:
        kw["ns"] = 40
    stepper, adt = build_dynamical_core(core, g, op, C, st, **kw)
    with torch.no_grad():
        for n in range(int(round(t_end / adt))):
            st = stepper.step(st, n * adt, None, lambda s, f: s)
    u, w = st["u"][:, 1, :], st["w"][:, 1, :]
    return {"u": 0.5 * (u[:-1] + u[1:]), "w": 0.5 * (w[:, :-1] + w[:, 1:]), "pi": st["pi"][:, 1, :],
            "th_v": st["th_v"][:, 1, :]}


def rates(sols, dx=250.0):
    c = int(1500.0 / dx)
    errs = {k: [float(torch.sqrt(torch.mean((b[k][c:-c, c:-c] - a[k][c:-c, c:-c]) ** 2)))
                for a, b in zip(sols[:-1], sols[1:])] for k in ("u", "w", "pi", "th_v")}
    return errs, {k: [math.log2(v[i] / v[i + 1]) for i in range(len(v) - 1)] for k, v in errs.items()}
