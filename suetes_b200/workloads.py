"""Synthetic workloads of the SISL benchmarks, built on the CUDA package.

* ``mountain_wave``: 3-D mountain-wave flow (the 256x256x80 configuration):
  dx = dy = 500 m, 80 levels over a 20 km lid with the stretched SLEVE
  coordinate (kappa 2.5, s = 4 km, n = 1.35; transforms.py:54-86), the ridge
  h(x) = 250 exp(-(x/5 km)^2) cos^2(pi x / 4 km) uniform in y
  (schaer_mountain_3d/run.py:83-85), U = 10 m/s, N = 0.01 1/s, dt = 8 s,
  alpha 0.5, sponge from 12 km, x relaxation over 4 km
  (schaer_mountain_3d/run.py:103-136).  No dataset is involved: the case
  is analytic.
* ``box_energy_objective``: the adjoint objective of the mountain-wave
  gradient runs -- the mean over the last steps of the box-averaged
  1/2 rho (u'^2 + v^2 + w^2) in the lee (x in [5, 25] km, z in [1, 6] km,
  all y), patterned on the box-energy objective of
  experiments/schaer_optimal_perturbation/run.py:138-144.
* ``bubble_ensemble``: the many-member configuration -- 32 warm-bubble
  members of uneven sizes (nx, ny in {64, 96, 128, 160}, nz in {40, 48, 64},
  dx = 50 m), amplitudes U[1, 3] K and centres jittered by +-300 m per axis,
  seeded with numpy's default_rng.
* ``rising_bubble``: 3-D dry warm bubble (64x64x48, 50 m, dt = 1 s,
  cos^2 bubble of 2 K, r = 1 km, 1.5 km above ground;
  cpu_gpu_short_scaling/run.py:38-55 in 3-D).
"""

import math

import torch

from .boundaries import x_relaxation
from .core import F32, F64
from .euler import Euler3D
from .geometry import RegionalGrid3D, StretchedSleveSimple
from .operators import CGridOperator3D
from .steppers import build_dynamical_core

CONSTANTS = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}


def ridge(x, y):
    return 250.0 * torch.exp(-(x / 5000.0) ** 2) * torch.cos(math.pi * x / 4000.0) ** 2 + 0.0 * y


def mountain_wave(nx=256, ny=256, nz=80, dtype=F32, device="cuda", solver_tol=1e-8, solver_maxiter=30,
                  solver_restart=30, solve_method="batched", dt=8.0, refine=True, flat=False):
    """``flat``: the same physics over flat terrain ("flat-then-SLEVE")."""
    h = (lambda x, y: 0.0 * x + 0.0 * y) if flat else ridge
    grid = RegionalGrid3D(nx, ny, nz, 500.0, 500.0, 20000.0 / nz, 45.0, 0.0, h_func=h,
                          transform=StretchedSleveSimple(2.5, 4000.0, 1.35), device=device)
    op = CGridOperator3D(grid)
    bgp = Euler3D(grid, op, CONSTANTS, dt=dt, N_bv=0.01)
    c = CONSTANTS
    rho = c["p0"] / (c["Rd"] * bgp.theta_bg) * bgp.pi_bg ** (c["cvd"] / c["Rd"])
    z = lambda *s: torch.zeros(*s, dtype=F64, device=grid.device)
    state = {"u": z(nx + 1, ny, nz) + 10.0, "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1),
             "eta_dot": z(nx, ny, nz + 1), "pi": bgp.pi_bg.clone(), "rho": rho, "th_v": bgp.theta_bg.clone()}
    stepper, _ = build_dynamical_core("sisl", grid, op, c, state, dt=dt, alpha=0.5, nu_div_factor=0.0,
                                      nu_h_factor=0.0, damp_height=12000.0, max_damp=0.5, N_bv=0.01,
                                      solver_tol=solver_tol, solver_maxiter=solver_maxiter,
                                      solver_restart=solver_restart, solve_method=solve_method)
    for k in ("u", "v", "w", "eta_dot", "u_prev", "v_prev", "w_prev", "eta_dot_prev", "tend_th_v_prev", "rho"):
        state[k] = state[k].to(dtype)
    stepper.implicit_solver.refine = bool(refine)
    bc = x_relaxation(grid, 4000.0, 10.0)
    return stepper, state, bc


def rising_bubble(nx=64, ny=64, nz=48, dx=50.0, amp=2.0, radius=1000.0, center=(0.0, 0.0, 1500.0), dtype=F64,
                  device="cuda", solver_tol=1e-10, solver_maxiter=100, solver_restart=100, solve_method="batched",
                  dt=1.0):
    grid = RegionalGrid3D(nx, ny, nz, dx, dx, dx, 0.0, 0.0, device=device)
    op = CGridOperator3D(grid)
    bgp = Euler3D(grid, op, CONSTANTS, dt=dt, N_bv=0.0)
    c = CONSTANTS
    X, Y, Zc = torch.meshgrid(grid.x_m, grid.y_m, grid.z_m, indexing="ij")
    r = torch.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Zc - center[2]) ** 2)
    th = bgp.theta_bg + torch.where(r < radius, amp * torch.cos(0.5 * math.pi * r / radius) ** 2, torch.zeros_like(r))
    rho = c["p0"] / (c["Rd"] * th) * bgp.pi_bg ** (c["cvd"] / c["Rd"])
    z = lambda *s: torch.zeros(*s, dtype=F64, device=grid.device)
    state = {"u": z(nx + 1, ny, nz), "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1), "eta_dot": z(nx, ny, nz + 1),
             "pi": bgp.pi_bg.clone(), "th_v": th, "rho": rho}
    stepper, _ = build_dynamical_core("sisl", grid, op, c, state, dt=dt, N_bv=0.0, nu_div_factor=0.0,
                                      nu_h_factor=0.0, solver_tol=solver_tol, solver_maxiter=solver_maxiter,
                                      solver_restart=solver_restart, solve_method=solve_method)
    for k in ("u", "v", "w", "eta_dot", "u_prev", "v_prev", "w_prev", "eta_dot_prev", "tend_th_v_prev", "rho"):
        state[k] = state[k].to(dtype)
    return stepper, state, None


def split_bubble(nx=256, ny=256, nz=64, dx=50.0, amp=2.0, radius=1000.0, center=(0.0, 0.0, 1500.0), dtype=F32,
                 device="cuda", dt=0.5, ns=12):
    """The 3-D warm bubble of ``rising_bubble`` (isentropic, flat, dx = dz)
    for the split-explicit core: ns acoustic steps per large step as in the
    reference's rising-bubble comparison (rising_bubble_3d/run.py:104-105),
    the factory's split-explicit stabilisation, damping above 2.5 km."""
    grid = RegionalGrid3D(nx, ny, nz, dx, dx, dx, 0.0, 0.0, device=device)
    op = CGridOperator3D(grid)
    bgp = Euler3D(grid, op, CONSTANTS, dt=dt, N_bv=0.0)
    c = CONSTANTS
    X, Y, Zc = torch.meshgrid(grid.x_m, grid.y_m, grid.z_m, indexing="ij")
    r = torch.sqrt((X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Zc - center[2]) ** 2)
    th = bgp.theta_bg + torch.where(r < radius, amp * torch.cos(0.5 * math.pi * r / radius) ** 2, torch.zeros_like(r))
    rho = c["p0"] / (c["Rd"] * th) * bgp.pi_bg ** (c["cvd"] / c["Rd"])
    z = lambda *s: torch.zeros(*s, dtype=F64, device=grid.device)
    state = {"u": z(nx + 1, ny, nz), "v": z(nx, ny + 1, nz), "w": z(nx, ny, nz + 1), "eta_dot": z(nx, ny, nz + 1),
             "pi": bgp.pi_bg.clone(), "th_v": th, "rho": rho}
    stepper, _ = build_dynamical_core("split-explicit", grid, op, c, state, dt=dt, ns=ns, N_bv=0.0,
                                      damp_height=2500.0, max_damp=0.05)
    for k in ("u", "v", "w", "eta_dot", "rho"):
        state[k] = state[k].to(dtype)
    return stepper, state


def box_energy_objective(stepper, num_steps, last=10, u_ref=10.0, x_box=(5000.0, 25000.0), z_box=(1000.0, 6000.0)):
    """``objective(n, state)`` for ``trajectory_vjp``: J = mean over the last
    ``last`` of ``num_steps`` states of the box-averaged kinetic energy of
    the perturbation wind, on mass points (perturbation-form state)."""
    from .core import fortran
    g = stepper.physics.grid
    op = stepper.physics.op
    X = g.x_m[:, None, None].expand(g.nx, g.ny, g.nz)
    Z = g.Z_m
    box = ((X >= x_box[0]) & (X <= x_box[1]) & (Z >= z_box[0]) & (Z <= z_box[1])).to(F64)
    count = float(box.sum())
    if count == 0.0:
        raise ValueError("the objective box holds no mass points")
    first = max(1, num_steps - last + 1)
    nterms = num_steps - first + 1
    cache = {}

    def objective(n, st):
        if n < first:
            return None
        dt_ = st["u"].dtype
        w8 = cache.get(dt_)
        if w8 is None:
            w8 = fortran(box, dtype=dt_) / (count * nterms)
            cache[dt_] = w8
        um = op.avg(st["u"], 0, "u", "m") - u_ref
        vm = op.avg(st["v"], 1, "v", "m")
        wm = op.avg(st["w"], 2, "w", "m")
        return (w8 * 0.5 * st["rho"] * (um * um + vm * vm + wm * wm)).sum()

    return objective


def bubble_ensemble(n_members=32, seed=0, dtype=F32, device="cuda", solver_tol=1e-7, solver_maxiter=30,
                    solver_restart=30, solve_method="incremental", dt=1.0):
    """[(stepper, state, bc, spec)] for the uneven-size bubble ensemble."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_members):
        nx = int(rng.choice([64, 96, 128, 160]))
        ny = int(rng.choice([64, 96, 128, 160]))
        nz = int(rng.choice([40, 48, 64]))
        amp = float(rng.uniform(1.0, 3.0))
        jit = rng.uniform(-300.0, 300.0, size=3)
        center = (float(jit[0]), float(jit[1]), 1500.0 + float(jit[2]))
        st, state, bc = rising_bubble(nx, ny, nz, dx=50.0, amp=amp, center=center, dtype=dtype, device=device,
                                      solver_tol=solver_tol, solver_maxiter=solver_maxiter,
                                      solver_restart=solver_restart, solve_method=solve_method, dt=dt)
        out.append((st, state, bc, {"nx": nx, "ny": ny, "nz": nz, "amp": amp, "center": center}))
    return out
