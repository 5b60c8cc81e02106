"""Oracle restatement of the grid, projection and vertical transforms.

Follows ``suetes/regional3d/geometry.py:13-272`` and
``suetes/shared/transforms.py:16-139``.  Test infrastructure only.
"""

import math

import torch

from . import DTYPE

OMEGA = 7.2921e-5  # geometry.py:202


def _t(x):
    return torch.as_tensor(x, dtype=DTYPE)


# ---------------------------------------------------------------------------
# Vertical transforms (transforms.py:16-139).  Called as T(xi, zeta, h, Lz).
# ---------------------------------------------------------------------------
class GalChenSigma:
    """z = h + zeta (Lz - h) / Lz  (transforms.py:16-22)."""

    def __call__(self, xi, zeta, h, Lz):
        return h + zeta * (Lz - h) / Lz


class HybridSigma:
    """transforms.py:25-35."""

    def __init__(self, scale_height=5000.0):
        self.scale_height = scale_height

    def __call__(self, xi, zeta, h, Lz):
        decay = (1.0 - zeta / Lz) * torch.exp(-zeta / self.scale_height)
        return zeta + h * decay


class SleveSimple:
    """transforms.py:38-51."""

    def __init__(self, scale_s=4000.0, scale_l=15000.0, n=1.35):
        self.ss, self.sl, self.n = scale_s, scale_l, n

    def __call__(self, xi, zeta, h, Lz):
        zeta_safe = torch.clamp(zeta, 0.0, Lz)
        b_s = torch.sinh((Lz - zeta_safe) / self.ss) / math.sinh(Lz / self.ss)
        b_s_safe = torch.clamp(b_s, 1e-8, 1.0)
        return zeta_safe + h * b_s_safe ** self.n


class StretchedSleveSimple:
    """transforms.py:54-86."""

    def __init__(self, stretch_kappa=2.5, scale_s=4000.0, n=1.35):
        self.kappa, self.ss, self.n = stretch_kappa, scale_s, n

    def __call__(self, xi, zeta, h, Lz):
        eta = zeta / Lz
        if abs(self.kappa) > 1e-5:
            zs = Lz * (torch.exp(self.kappa * eta) - 1.0) / (math.exp(self.kappa) - 1.0)
        else:
            zs = zeta
        zs = torch.clamp(zs, 0.0, Lz)
        b_s = torch.sinh((Lz - zs) / self.ss) / math.sinh(Lz / self.ss)
        b_s_safe = torch.clamp(b_s, 1e-8, 1.0)
        return zs + h * b_s_safe ** self.n


# ---------------------------------------------------------------------------
# Projection (geometry.py:13-87)
# ---------------------------------------------------------------------------
class ObliqueStereographic:
    def __init__(self, lat_center, lon_center, R_earth=6371229.0, eps=1e-15):
        self.phi_c = math.radians(lat_center)
        self.lam_c = math.radians(lon_center)
        self.R = R_earth
        self.eps = eps

    def get_map_factor(self, x, y):  # geometry.py:35-52
        return 1.0 + (x ** 2 + y ** 2) / (4.0 * self.R ** 2)

    def get_lat_lon(self, x, y):  # geometry.py:54-87
        rho = torch.sqrt(x ** 2 + y ** 2)
        rho = torch.where(rho == 0, torch.full_like(rho, self.eps), rho)
        c = 2.0 * torch.atan(rho / (2.0 * self.R))
        sin_c, cos_c = torch.sin(c), torch.cos(c)
        sp, cpc = math.sin(self.phi_c), math.cos(self.phi_c)
        lat = torch.asin(cos_c * sp + (y * sin_c * cpc) / rho)
        lon = self.lam_c + torch.atan2(x * sin_c, rho * cpc * cos_c - y * sp * sin_c)
        return torch.rad2deg(lat), torch.rad2deg(lon)


def _h_eval(h_func, x, y):
    h = h_func(x, y)
    if not torch.is_tensor(h):
        h = torch.full_like(x, float(h))
    return torch.broadcast_to(h.to(DTYPE), x.shape)


class RegionalGrid3D:
    """Grid, map factors, Coriolis and terrain metrics (geometry.py:141-272).

    ``h_func(x, y)`` and ``transform`` receive float64 torch tensors.
    """

    def __init__(self, nx, ny, nz, dx, dy, dz, lat_center, lon_center,
                 h_func=None, transform=None, eps=1e-15):
        self.shape = (nx, ny, nz)
        self.delta = (dx, dy, dz)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx, self.dy, self.dz = dx, dy, dz
        self.lat_c, self.lon_c = lat_center, lon_center
        Lx, Ly = nx * dx, ny * dy
        self.Lz = nz * dz

        self.x_c = torch.arange(nx + 1, dtype=DTYPE) * dx - Lx / 2.0
        self.y_c = torch.arange(ny + 1, dtype=DTYPE) * dy - Ly / 2.0
        self.z_c = torch.arange(nz + 1, dtype=DTYPE) * dz
        self.x_m = 0.5 * (self.x_c[:-1] + self.x_c[1:])
        self.y_m = 0.5 * (self.y_c[:-1] + self.y_c[1:])
        self.z_m = 0.5 * (self.z_c[:-1] + self.z_c[1:])

        mg = lambda *a: torch.meshgrid(*a, indexing="ij")
        Xm2, Ym2 = mg(self.x_m, self.y_m)
        Xu2, Yu2 = mg(self.x_c, self.y_m)
        Xv2, Yv2 = mg(self.x_m, self.y_c)

        self.proj = ObliqueStereographic(lat_center, lon_center, eps=eps)
        self.m_factors = {
            "m": self.proj.get_map_factor(Xm2, Ym2),
            "u": self.proj.get_map_factor(Xu2, Yu2),
            "v": self.proj.get_map_factor(Xv2, Yv2),
            "w": self.proj.get_map_factor(Xm2, Ym2),
        }
        # geometry.py:198-199
        self.dm_dx_m = Xm2 / (2.0 * self.proj.R ** 2)
        self.dm_dy_m = Ym2 / (2.0 * self.proj.R ** 2)
        # geometry.py:202-209
        lat_m, _ = self.proj.get_lat_lon(Xm2, Ym2)
        lat_u, _ = self.proj.get_lat_lon(Xu2, Yu2)
        lat_v, _ = self.proj.get_lat_lon(Xv2, Yv2)
        self.f_m = 2.0 * OMEGA * torch.sin(torch.deg2rad(lat_m))
        self.f_u = 2.0 * OMEGA * torch.sin(torch.deg2rad(lat_u))
        self.f_v = 2.0 * OMEGA * torch.sin(torch.deg2rad(lat_v))

        self.h_func = h_func if h_func is not None else (lambda x, y: 0.0)
        self.transform_op = transform if transform is not None else GalChenSigma()

        Xi_m, Yi_m, Ze_m = mg(self.x_m, self.y_m, self.z_m)
        Xi_u, Yi_u, Ze_u = mg(self.x_c, self.y_m, self.z_m)
        Xi_v, Yi_v, Ze_v = mg(self.x_m, self.y_c, self.z_m)
        Xi_w, Yi_w, Ze_w = mg(self.x_m, self.y_m, self.z_c)

        def apply_transform(xi, eta, zeta):  # geometry.py:226-229
            h = _h_eval(self.h_func, xi, eta)
            return self.transform_op(xi, zeta, h, self.Lz)

        self.Z_m = apply_transform(Xi_m, Yi_m, Ze_m)
        self.Z_u = apply_transform(Xi_u, Yi_u, Ze_u)
        self.Z_v = apply_transform(Xi_v, Yi_v, Ze_v)
        self.Z_w = apply_transform(Xi_w, Yi_w, Ze_w)

        # geometry.py:242-252
        self.dz_m_full = self.Z_w[:, :, 1:] - self.Z_w[:, :, :-1]
        bot = self.Z_m[:, :, 0] - (self.Z_m[:, :, 1] - self.Z_m[:, :, 0])
        top = self.Z_m[:, :, -1] + (self.Z_m[:, :, -1] - self.Z_m[:, :, -2])
        Zp = torch.cat([bot[..., None], self.Z_m, top[..., None]], dim=-1)
        self.dz_w_full = Zp[:, :, 1:] - Zp[:, :, :-1]
        # geometry.py:257-261 (edge-padded centred differences)
        Zx = torch.cat([self.Z_w[:1], self.Z_w, self.Z_w[-1:]], dim=0)
        self.z_xi_w = (Zx[2:] - Zx[:-2]) / (2.0 * dx)
        Zy = torch.cat([self.Z_w[:, :1], self.Z_w, self.Z_w[:, -1:]], dim=1)
        self.z_eta_w = (Zy[:, 2:] - Zy[:, :-2]) / (2.0 * dy)

        dz_min = float(self.dz_m_full.min())  # geometry.py:264-272
        if dz_min <= 0.0:
            raise ValueError(
                f"Grid Tangling Detected! Minimum dz is {dz_min:.2f} m.\n"
                "The 3D topography is too steep. Smooth the terrain or increase Lz."
            )
