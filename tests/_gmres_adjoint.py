"""Adjoint sensitivity to the GMRES solve (verification/gmres_adjoint_convergence.py).

The float64 gradient of 0.5 sum(rho w_m^2 + 0.1 theta'^2) dx dy dz after
T = 30 s with respect to the initial theta', on the 40 x 3 x 20 warm bubble
of :50-78 (dx = dz = 150 m, 3 K bubble 1500 m up, sponge above 7.5 km of
strength 0.05, alpha 0.55, restart 40), with the forward and transposed
solves capped at `maxiter` restart cycles, against the same gradient at
tol 1e-12 (:80-107, :143-166).  The background is built once from the
initial state and held fixed."""

import math

import torch

C = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}


def _case(device, nx=40, ny=3, nz=20, dx=150.0):
    from suetes_b200 import RegionalGrid3D, CGridOperator3D, Euler3D
    g = RegionalGrid3D(nx, ny, nz, dx, dx, dx, 0.0, 0.0, device=device)
    op = CGridOperator3D(g)
    ph = Euler3D(g, op, C, dt=1.0, N_bv=0.0)
    th_bg, pi_bg = ph.theta_bg.double().cpu(), ph.pi_bg.double().cpu()
    z = lambda *s: torch.zeros(*s, dtype=torch.float64)
    x, _, zz = torch.meshgrid(g.x_m.double().cpu(), g.y_m.double().cpu(), g.z_m.double().cpu(), indexing="ij")
    r = torch.sqrt(x ** 2 + (zz - 1500.0) ** 2)
    bubble = torch.where(r <= 1000.0, 3.0 * torch.cos(0.5 * math.pi * r / 1000.0) ** 2, torch.zeros_like(r))
    th = th_bg + bubble
    st = {"u": z(nx + 1, ny, nz), "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1), "eta_dot": z(nx, ny, nz + 1),
          "pi": pi_bg.clone(), "th_v": th, "rho": C["p0"] / (C["Rd"] * th) * pi_bg ** (C["cvd"] / C["Rd"])}
    return g, op, {k: v.to(device) for k, v in st.items()}


def gradient(dt, maxiter, tol, device="cuda", T=30.0):
    """(J, dJ/dtheta'_0) with both solves capped at `maxiter` cycles."""
    from suetes_b200 import build_dynamical_core
    from suetes_b200.adjoint import trajectory_vjp
    g, op, st = _case(device)
    stepper, adt = build_dynamical_core("sisl", g, op, C, dict(st), dt=dt, solver_tol=tol, solver_maxiter=maxiter,
                                        solver_restart=40, damp_height=7500.0, max_damp=0.05, alpha=0.55)
    n = max(1, int(T / dt))
    vol = g.dx * g.dy * g.dz
    th_bg = stepper.physics.theta_bg.to(device)

    def objective(k, s):
        if k != n:
            return None
        wc = 0.5 * (s["w"][:, :, :-1] + s["w"][:, :, 1:])
        thp = s["th_p"] + th_bg - 300.0
        return 0.5 * (s["rho"] * wc ** 2 + 0.1 * thp ** 2).sum() * vol

    J, gr = trajectory_vjp(stepper, st, n, objective, wrt=("th_p",))
    return float(J), gr["th_p"].double().cpu()
