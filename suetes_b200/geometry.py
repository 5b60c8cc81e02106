"""Grid, map projection and vertical transforms (set-up, float64).

Mirrors ``RegionalGrid3D`` / ``ObliqueStereographic`` of the reference
(``suetes/regional3d/geometry.py:13-272``) and the vertical transforms of
``suetes/shared/transforms.py:16-139``.  Everything here runs once per grid
with torch float64 tensors on the grid's device; the arrays become inputs of
the CUDA core (``sisl_core_create``).  ``h_func(x, y)`` and the transforms
receive torch float64 tensors.
"""

import math

import torch

F64 = torch.float64
OMEGA = 7.2921e-5


def default_device():
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


class GalChenSigma:
    """z = h + zeta (Lz - h) / Lz  (transforms.py:16-22)."""

    def __call__(self, xi, zeta, h, Lz):
        return h + zeta * (Lz - h) / Lz


class HybridSigma:
    """Exponentially decaying terrain influence (transforms.py:25-35)."""

    def __init__(self, scale_height=5000.0):
        self.scale_height = scale_height

    def __call__(self, xi, zeta, h, Lz):
        return zeta + h * (1.0 - zeta / Lz) * torch.exp(-zeta / self.scale_height)


class SleveSimple:
    """Single-scale SLEVE (transforms.py:38-51)."""

    def __init__(self, scale_s=4000.0, scale_l=15000.0, n=1.35):
        self.ss, self.sl, self.n = scale_s, scale_l, n

    def __call__(self, xi, zeta, h, Lz):
        zs = torch.clamp(zeta, 0.0, Lz)
        b = torch.clamp(torch.sinh((Lz - zs) / self.ss) / math.sinh(Lz / self.ss), 1e-8, 1.0)
        return zs + h * b ** self.n


class StretchedSleveSimple:
    """SLEVE with exponential low-level stretching (transforms.py:54-86)."""

    def __init__(self, stretch_kappa=2.5, scale_s=4000.0, n=1.35):
        self.kappa, self.ss, self.n = stretch_kappa, scale_s, n

    def __call__(self, xi, zeta, h, Lz):
        e = zeta / Lz
        zs = (Lz * (torch.exp(self.kappa * e) - 1.0) / (math.exp(self.kappa) - 1.0)
              if abs(self.kappa) > 1e-5 else zeta)
        zs = torch.clamp(zs, 0.0, Lz)
        b = torch.clamp(torch.sinh((Lz - zs) / self.ss) / math.sinh(Lz / self.ss), 1e-8, 1.0)
        return zs + h * b ** self.n


class ObliqueStereographic:
    """Conformal projection with isotropic map factor (geometry.py:13-87)."""

    def __init__(self, lat_center, lon_center, R_earth=6371229.0, eps=1e-15):
        self.phi_c, self.lam_c = math.radians(lat_center), math.radians(lon_center)
        self.R, self.eps = R_earth, eps

    def get_map_factor(self, x, y):
        return 1.0 + (x * x + y * y) / (4.0 * self.R ** 2)

    def get_lat_lon(self, x, y):
        rho = torch.sqrt(x * x + y * y)
        rho = torch.where(rho == 0, torch.full_like(rho, self.eps), rho)
        c = 2.0 * torch.atan(rho / (2.0 * self.R))
        sp, cph = math.sin(self.phi_c), math.cos(self.phi_c)
        lat = torch.asin(torch.cos(c) * sp + y * torch.sin(c) * cph / rho)
        lon = self.lam_c + torch.atan2(x * torch.sin(c), rho * cph * torch.cos(c) - y * sp * torch.sin(c))
        return torch.rad2deg(lat), torch.rad2deg(lon)


class RegionalGrid3D:
    """Arakawa-C / Lorenz grid with terrain-following metrics (geometry.py:127-272)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, lat_center, lon_center, h_func=None, transform=None,
                 eps=1e-15, device=None):
        if min(nx, ny, nz) < 2:
            raise ValueError("nx, ny and nz must be at least 2")
        dev = torch.device(device) if device is not None else default_device()
        self.device = dev
        self.shape, self.delta = (nx, ny, nz), (dx, dy, dz)
        self.nx, self.ny, self.nz, self.dx, self.dy, self.dz = nx, ny, nz, dx, dy, dz
        self.lat_c, self.lon_c = lat_center, lon_center
        Lx, Ly = nx * dx, ny * dy
        self.Lz = nz * dz
        ar = lambda n: torch.arange(n, dtype=F64, device=dev)
        self.x_c = ar(nx + 1) * dx - Lx / 2.0
        self.y_c = ar(ny + 1) * dy - Ly / 2.0
        self.z_c = ar(nz + 1) * dz
        self.x_m = 0.5 * (self.x_c[:-1] + self.x_c[1:])
        self.y_m = 0.5 * (self.y_c[:-1] + self.y_c[1:])
        self.z_m = 0.5 * (self.z_c[:-1] + self.z_c[1:])
        mg = lambda *a: torch.meshgrid(*a, indexing="ij")
        Xm, Ym = mg(self.x_m, self.y_m)
        Xu, Yu = mg(self.x_c, self.y_m)
        Xv, Yv = mg(self.x_m, self.y_c)
        self.proj = ObliqueStereographic(lat_center, lon_center, eps=eps)
        mf = self.proj.get_map_factor
        self.m_factors = {"m": mf(Xm, Ym), "u": mf(Xu, Yu), "v": mf(Xv, Yv), "w": mf(Xm, Ym)}
        self.dm_dx_m = Xm / (2.0 * self.proj.R ** 2)
        self.dm_dy_m = Ym / (2.0 * self.proj.R ** 2)
        self.f_m = 2.0 * OMEGA * torch.sin(torch.deg2rad(self.proj.get_lat_lon(Xm, Ym)[0]))
        self.f_u = 2.0 * OMEGA * torch.sin(torch.deg2rad(self.proj.get_lat_lon(Xu, Yu)[0]))
        self.f_v = 2.0 * OMEGA * torch.sin(torch.deg2rad(self.proj.get_lat_lon(Xv, Yv)[0]))
        self.h_func = h_func if h_func is not None else (lambda x, y: 0.0)
        self.transform_op = transform if transform is not None else GalChenSigma()

        def Z(xs, ys, zs):
            X, Y, Ze = mg(xs, ys, zs)
            h = self.h_func(X, Y)
            h = torch.broadcast_to(torch.as_tensor(h, dtype=F64, device=dev), X.shape)
            return self.transform_op(X, Ze, h, self.Lz)

        self.Z_m = Z(self.x_m, self.y_m, self.z_m)
        self.Z_u = Z(self.x_c, self.y_m, self.z_m)
        self.Z_v = Z(self.x_m, self.y_c, self.z_m)
        self.Z_w = Z(self.x_m, self.y_m, self.z_c)
        self.dz_m_full = self.Z_w[:, :, 1:] - self.Z_w[:, :, :-1]
        bot = self.Z_m[:, :, :1] - (self.Z_m[:, :, 1:2] - self.Z_m[:, :, :1])
        top = self.Z_m[:, :, -1:] + (self.Z_m[:, :, -1:] - self.Z_m[:, :, -2:-1])
        Zp = torch.cat([bot, self.Z_m, top], dim=2)
        self.dz_w_full = Zp[:, :, 1:] - Zp[:, :, :-1]
        Zx = torch.cat([self.Z_w[:1], self.Z_w, self.Z_w[-1:]], dim=0)
        self.z_xi_w = (Zx[2:] - Zx[:-2]) / (2.0 * dx)
        Zy = torch.cat([self.Z_w[:, :1], self.Z_w, self.Z_w[:, -1:]], dim=1)
        self.z_eta_w = (Zy[:, 2:] - Zy[:, :-2]) / (2.0 * dy)
        dz_min = float(self.dz_m_full.min())
        if dz_min <= 0.0:
            raise ValueError(f"Grid Tangling Detected! Minimum dz is {dz_min:.2f} m.\n"
                             "The 3D topography is too steep. Smooth the terrain or increase Lz.")

    def shape_of(self, loc):
        return (self.nx + (loc == "u"), self.ny + (loc == "v"), self.nz + (loc == "w"))
