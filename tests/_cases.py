"""Shared test cases: the same grids and states built for the oracle (CPU,
float64) and for the CUDA package.  Grids follow the reference tests
(tests/test_dynamical_core_3d.py:20-40, tests/test_core_formula_regressions.py:45-76)."""

import math

import torch

C = {"g": 9.81, "cp": 1004.0, "Rd": 287.0, "cvd": 717.0, "p0": 100000.0}


def mountain(x, y):
    return 1500.0 * torch.exp(-(x ** 2 + y ** 2) / (5000.0 ** 2))


def ridge(x, y):
    return 250.0 * torch.exp(-(x / 5000.0) ** 2) * torch.cos(math.pi * x / 4000.0) ** 2 + 0.0 * y


def build(pkg, nx, ny, nz, dx, dy, dz, lat=45.0, lon=0.0, h=None, transform=None, periodic=(), device=None,
          **euler_kw):
    if pkg == "oracle":
        from oracle.grid import RegionalGrid3D
        from oracle.ops import CGridOperator3D
        from oracle.euler import Euler3D
        g = RegionalGrid3D(nx, ny, nz, dx, dy, dz, lat, lon, h_func=h, transform=transform)
    else:
        from suetes_b200 import RegionalGrid3D, CGridOperator3D, Euler3D
        g = RegionalGrid3D(nx, ny, nz, dx, dy, dz, lat, lon, h_func=h, transform=transform, device=device)
    op = CGridOperator3D(g, periodic_axes=periodic)
    ph = Euler3D(g, op, C, **euler_kw)
    return g, op, ph


def random_fields(shapes, seed, scales, dtype=torch.float64):
    gen = torch.Generator().manual_seed(seed)
    return {k: (torch.rand(shapes[k], generator=gen, dtype=torch.float64) - 0.5) * 2 * scales[k]
            for k in shapes}


def shapes5(nx, ny, nz):
    return {"u": (nx + 1, ny, nz), "v": (nx, ny + 1, nz), "w": (nx, ny, nz + 1), "pi": (nx, ny, nz),
            "eta_dot": (nx, ny, nz + 1)}


def to_cuda(d, dtype=torch.float64):
    return {k: (v.to("cuda", dtype) if torch.is_tensor(v) else v) for k, v in d.items()}


def to_cpu(d):
    return {k: (v.detach().double().cpu() if torch.is_tensor(v) else v) for k, v in d.items()}


def rel_l2(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))


def max_abs(a, b):
    return float((a.detach().double().cpu() - b.detach().double().cpu()).abs().max())
