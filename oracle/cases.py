"""Oracle-side builders of the benchmark cases: TEST INFRASTRUCTURE ONLY.

The same analytic cases as ``suetes_b200.workloads``, built on the float64
CPU oracle, for the GPU-vs-oracle parity tests and the CPU legs of the
bench:

* ``rising_bubble``: the 3-D dry warm bubble (64x64x48, dx = dy = dz = 50 m,
  flat terrain, isentropic 300 K, cos^2 bubble of 2 K and radius 1 km
  centred 1.5 km above ground, zero wind, dt = 1 s; the 3-D form of
  benchmarks/performance/cpu_gpu_short_scaling/run.py:38-55 and
  benchmarks/physical/rising_bubble_3d/run.py:87-91), GMRES restart and
  maxiter 100 (the factory defaults, steppers.py:47-49).
* ``mountain_wave``: the 3-D mountain wave over the stretched SLEVE
  coordinate (dx = dy = 500 m, 20 km lid, kappa 2.5, s = 4 km, n = 1.35),
  the ridge 250 exp(-(x/5 km)^2) cos^2(pi x / 4 km) uniform in y
  (schaer_mountain_3d/run.py:83-85), U = 10 m/s, N = 0.01 1/s, dt = 8 s,
  alpha 0.5, sponge from 12 km, and the cos^2 x relaxation over 4 km as its
  bc_fn (schaer_mountain_3d/run.py:104-126).
"""

import math

import torch

from . import DTYPE
from .euler import Euler3D
from .grid import RegionalGrid3D, StretchedSleveSimple
from .ops import CGridOperator3D
from .steppers import build_dynamical_core

CONSTANTS = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}


def _zeros(*s):
    return torch.zeros(*s, dtype=DTYPE)


def rising_bubble(nx=64, ny=64, nz=48, dx=50.0, amp=2.0, radius=1000.0, center=(0.0, 0.0, 1500.0),
                  solver_tol=1e-10, solver_maxiter=100, solver_restart=100, dt=1.0):
    """(stepper, state, bc_fn) of the warm bubble; bc_fn is the identity."""
    c = CONSTANTS
    g = RegionalGrid3D(nx, ny, nz, dx, dx, dx, 0.0, 0.0)
    op = CGridOperator3D(g)
    bgp = Euler3D(g, op, c, dt=dt, N_bv=0.0)
    X, Y, Z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    r = torch.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Z - center[2]) ** 2)
    th = bgp.theta_bg + torch.where(r < radius, amp * torch.cos(0.5 * math.pi * r / radius) ** 2,
                                    torch.zeros_like(r))
    rho = c["p0"] / (c["Rd"] * th) * bgp.pi_bg ** (c["cvd"] / c["Rd"])
    st = {"u": _zeros(nx + 1, ny, nz), "v": _zeros(nx, ny + 1, nz), "w": _zeros(nx, ny, nz + 1),
          "eta_dot": _zeros(nx, ny, nz + 1), "pi": bgp.pi_bg.clone(), "th_v": th, "rho": rho}
    stepper, _ = build_dynamical_core("sisl", g, op, c, st, dt=dt, N_bv=0.0, nu_div_factor=0.0,
                                      nu_h_factor=0.0, solver_tol=solver_tol, solver_maxiter=solver_maxiter,
                                      solver_restart=solver_restart)
    return stepper, st, (lambda s, forcing: s)


def mountain_wave(nx, ny, nz, solver_tol=1e-8, solver_maxiter=30, solver_restart=30, dt=8.0,
                  solve_method="batched"):
    """(stepper, state, bc_fn) of the mountain wave on an nx x ny x nz grid
    with the workload's spacing, terrain, physics and x relaxation."""
    c = CONSTANTS
    ridge = lambda x, y: 250.0 * torch.exp(-(x / 5000.0) ** 2) * torch.cos(math.pi * x / 4000.0) ** 2 + 0.0 * y
    g = RegionalGrid3D(nx, ny, nz, 500.0, 500.0, 20000.0 / nz, 45.0, 0.0, h_func=ridge,
                       transform=StretchedSleveSimple(2.5, 4000.0, 1.35))
    op = CGridOperator3D(g)
    bgp = Euler3D(g, op, c, dt=dt, N_bv=0.01)
    rho = c["p0"] / (c["Rd"] * bgp.theta_bg) * bgp.pi_bg ** (c["cvd"] / c["Rd"])
    st = {"u": _zeros(nx + 1, ny, nz) + 10.0, "v": _zeros(nx, ny + 1, nz), "w": _zeros(nx, ny, nz + 1),
          "eta_dot": _zeros(nx, ny, nz + 1), "pi": bgp.pi_bg.clone(), "rho": rho, "th_v": bgp.theta_bg.clone()}
    stepper, _ = build_dynamical_core("sisl", g, op, c, st, dt=dt, alpha=0.5, nu_div_factor=0.0, nu_h_factor=0.0,
                                      damp_height=12000.0, max_damp=0.5, N_bv=0.01, solver_tol=solver_tol,
                                      solver_maxiter=solver_maxiter, solver_restart=solver_restart)
    stepper.implicit_solver.solve_method = solve_method
    n = round(4000.0 / g.dx)
    i = torch.arange(nx, dtype=DTYPE)
    d = torch.minimum(i, nx - 1 - i)
    mask = torch.where(d < n, torch.cos(0.5 * math.pi * d / n) ** 2, torch.zeros_like(d))[:, None, None]
    ph = stepper.physics

    def bc(s, forcing):  # schaer_mountain_3d/run.py:111-126
        out = dict(s)
        for k in ("u", "v", "th_v", "pi", "rho"):
            m = torch.cat([mask, mask[-1:]], dim=0) if k == "u" else mask
            ext = {"u": torch.full_like(s["u"], 10.0), "v": torch.zeros_like(s["v"]), "th_v": ph.theta_bg,
                   "pi": ph.pi_bg, "rho": ph.bg_state_ref()["rho"]}[k]
            out[k] = (1.0 - m) * s[k] + m * ext
        return out

    return stepper, st, bc
