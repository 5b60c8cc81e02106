"""Oracle restatement of ``Euler3D`` and ``HyperFilter``.

Follows ``suetes/regional3d/euler.py:13-439`` and
``suetes/regional3d/diffusion.py:80-173``.  Test infrastructure only.
"""

import math

import torch

from . import DTYPE


def jnp_interp(x, xp, fp):
    """``jnp.interp(x, xp, fp)`` with clamped ends (used at euler.py:82)."""
    n = xp.shape[0]
    i = torch.clamp(torch.searchsorted(xp, x.reshape(-1).contiguous(), right=True), 1, n - 1)
    i = i.reshape(x.shape)
    df = fp[i] - fp[i - 1]
    dxx = xp[i] - xp[i - 1]
    delta = x - xp[i - 1]
    tiny = torch.finfo(DTYPE).eps * 2.0 ** -52
    dx0 = dxx.abs() <= tiny
    f = torch.where(dx0, fp[i - 1], fp[i - 1] + (delta / torch.where(dx0, torch.ones_like(dxx), dxx)) * df)
    f = torch.where(x < xp[0], fp[0], f)
    f = torch.where(x > xp[-1], fp[-1], f)
    return f


class HyperFilter:
    """4th-order terrain-aware hyperdiffusion (diffusion.py:80-173)."""

    def __init__(self, grid, operators, nu_h=1e6, nu_v=1e6):
        self.grid, self.op, self.nu_h, self.nu_v = grid, operators, nu_h, nu_v

    def _cartesian_horizontal_laplacian(self, f_m, bg):  # diffusion.py:93-129
        op, g = self.op, self.grid
        df_dxi_u = op.diff(f_m, 0, "m", "u")
        df_dz_m = op.avg(op.diff(f_m, 2, "m", "w") * (g.dz / bg["dz_w_full"]), 2, "w", "m")
        df_dz_u = op.avg(df_dz_m, 0, "m", "u")
        z_xi_u = op.diff(g.Z_m, 0, "m", "u")
        Gx_u = df_dxi_u - z_xi_u * df_dz_u
        df_deta_v = op.diff(f_m, 1, "m", "v")
        df_dz_v = op.avg(df_dz_m, 1, "m", "v")
        z_eta_v = op.diff(g.Z_m, 1, "m", "v")
        Gy_v = df_deta_v - z_eta_v * df_dz_v
        dGx_dxi_m = op.diff(Gx_u, 0, "u", "m")
        Gx_m = op.avg(Gx_u, 0, "u", "m")
        dGx_dz_w = op.diff(Gx_m, 2, "m", "w") * (g.dz / bg["dz_w_full"])
        dGx_dz_m = op.avg(dGx_dz_w, 2, "w", "m")
        z_xi_m = op.avg(z_xi_u, 0, "u", "m")
        div_Gx = dGx_dxi_m - z_xi_m * dGx_dz_m
        dGy_deta_m = op.diff(Gy_v, 1, "v", "m")
        Gy_m = op.avg(Gy_v, 1, "v", "m")
        dGy_dz_w = op.diff(Gy_m, 2, "m", "w") * (g.dz / bg["dz_w_full"])
        dGy_dz_m = op.avg(dGy_dz_w, 2, "w", "m")
        z_eta_m = op.avg(z_eta_v, 1, "v", "m")
        div_Gy = dGy_deta_m - z_eta_m * dGy_dz_m
        return div_Gx + div_Gy

    def _vertical_laplacian(self, f_m, bg):  # diffusion.py:131-134
        op, g = self.op, self.grid
        df_dz_w = op.diff(f_m, 2, "m", "w") * (g.dz / bg["dz_w_full"])
        return op.diff(df_dz_w, 2, "w", "m") * (g.dz / bg["dz_m_full"])

    def get_tendencies(self, state_prime, bg_precomputed):  # diffusion.py:136-173
        op, bg = self.op, bg_precomputed
        out = {}
        for k in ("u", "v", "w", "th_v"):
            if k in state_prime or (k == "th_v" and "th_v_prime_m" in state_prime):
                if k == "u":
                    f_m = op.avg(state_prime["u"], 0, "u", "m")
                elif k == "v":
                    f_m = op.avg(state_prime["v"], 1, "v", "m")
                elif k == "w":
                    f_m = op.avg(state_prime["w"], 2, "w", "m")
                elif "th_v" in state_prime:
                    f_m = state_prime["th_v"] - bg["th_v"]
                else:
                    f_m = state_prime["th_v_prime_m"]
                lap1_h = self._cartesian_horizontal_laplacian(f_m, bg)
                lap1_v = self._vertical_laplacian(f_m, bg)
                hyper_h = -self.nu_h * self._cartesian_horizontal_laplacian(lap1_h, bg)
                hyper_v = -self.nu_v * self._vertical_laplacian(lap1_v, bg)
                tend_m = hyper_h + hyper_v
                if k == "u":
                    out["u"] = op.avg(tend_m, 0, "m", "u")
                elif k == "v":
                    out["v"] = op.avg(tend_m, 1, "m", "v")
                elif k == "w":
                    out["w"] = op.avg(tend_m, 2, "m", "w")
                else:
                    out["th_v"] = tend_m
        return out


class Euler3D:
    """Background state, tendencies and Helmholtz matvec (euler.py:13-439)."""

    def __init__(self, grid, operators, constants, dt, initial_era5_state=None,
                 N_bv=0.01, damp_height=20000.0, max_damp=0.5,
                 nu_div_factor=0.8, nu_h_factor=0.1, physics_suite=None,
                 interior_mask=None):
        self.grid, self.op, self.c, self.dt = grid, operators, constants, dt
        max_nu_div = grid.dx ** 2 / (4.0 * dt)  # euler.py:62-67
        max_nu_h = grid.dx ** 4 / (64.0 * dt)
        self.nu_div = nu_div_factor * max_nu_div
        self.nu_h = nu_h_factor * max_nu_h
        self.physics_suite = physics_suite
        self.interior_mask = interior_mask
        Z_m = grid.Z_m
        g, cp = constants["g"], constants["cp"]
        if initial_era5_state is not None:  # euler.py:76-85
            z_1d = Z_m.mean(dim=(0, 1))
            th_1d = torch.as_tensor(initial_era5_state["th_v"], dtype=DTYPE).mean(dim=(0, 1))
            self.theta_bg = jnp_interp(Z_m, z_1d, th_1d)
            pi_anchor_top = torch.as_tensor(initial_era5_state["pi"], dtype=DTYPE)[:, :, -1].mean()
        else:  # euler.py:86-96
            self.theta_0 = 300.0
            if N_bv > 0.0:
                self.theta_bg = self.theta_0 * torch.exp((N_bv ** 2 / g) * Z_m)
            else:
                self.theta_bg = self.theta_0 * torch.ones_like(Z_m)
            z_max = Z_m.max()
            if N_bv > 0.0:
                pi_anchor_top = 1.0 + (g ** 2 / (cp * self.theta_0 * N_bv ** 2)) * (
                    torch.exp(-N_bv ** 2 * z_max / g) - 1.0)
            else:
                pi_anchor_top = 1.0 - (g / (cp * self.theta_0)) * z_max
        # euler.py:100-112 hydrostatic integration from the lid
        delta_z = Z_m[:, :, 1:] - Z_m[:, :, :-1]
        th_w = 0.5 * (self.theta_bg[:, :, 1:] + self.theta_bg[:, :, :-1])
        delta_pi = -(g * delta_z) / (cp * th_w)
        rev = torch.flip(torch.cumsum(torch.flip(delta_pi, dims=[-1]), dim=-1), dims=[-1])
        top = torch.full((grid.nx, grid.ny, 1), float(pi_anchor_top), dtype=DTYPE)
        self.pi_bg = torch.cat([top - rev, top], dim=2)
        # euler.py:114-121
        zw, zt = grid.Z_w, grid.Lz
        self.tau_damp = torch.where(
            zw > damp_height,
            max_damp * 0.5 * (1.0 + torch.tanh(math.pi * (zw - damp_height) / (zt - damp_height) - math.pi / 2)),
            torch.zeros_like(zw))
        self.diffusion = HyperFilter(grid, operators, nu_h=self.nu_h, nu_v=0.0)

    def bg_state_ref(self):
        """Background dict built inside ``step`` (steppers.py:769-774)."""
        c = self.c
        rho = c["p0"] / (c["Rd"] * self.theta_bg) * self.pi_bg ** (c["cvd"] / c["Rd"])
        return {"rho": rho, "pi": self.pi_bg, "th_v": self.theta_bg}

    def precompute_bg(self, bg_state):  # euler.py:127-160
        op, g = self.op, self.grid
        th, rho, pi = bg_state["th_v"], bg_state["rho"], bg_state["pi"]
        return {
            "th_v_u": op.avg(th, 0, "m", "u"), "th_v_v": op.avg(th, 1, "m", "v"),
            "th_v_w": op.avg(th, 2, "m", "w"),
            "rho_u": op.avg(rho, 0, "m", "u"), "rho_v": op.avg(rho, 1, "m", "v"),
            "rho_w": op.avg(rho, 2, "m", "w"),
            "dz_m_full": g.dz_m_full, "dz_w_full": g.dz_w_full,
            "dz_u": op.avg(g.dz_m_full, 0, "m", "u"), "dz_v": op.avg(g.dz_m_full, 1, "m", "v"),
            "C_pi": (self.c["Rd"] / self.c["cvd"]) * (pi / (rho * th)),
            "pi_bg": pi, "th_v": th,
        }

    def nonlinear_pi_tendency(self, state_prime, th_v_prime, bg):  # euler.py:162-186
        op, g = self.op, self.grid
        tu = op.avg(th_v_prime, 0, "m", "u")
        tv = op.avg(th_v_prime, 1, "m", "v")
        tw = op.avg(th_v_prime, 2, "m", "w")
        m_u = g.m_factors["u"][..., None]
        m_v = g.m_factors["v"][..., None]
        m_m = g.m_factors["m"][..., None]
        fx = state_prime["u"] * bg["rho_u"] * tu * bg["dz_u"] / m_u
        fy = state_prime["v"] * bg["rho_v"] * tv * bg["dz_v"] / m_v
        fz = state_prime["eta_dot"] * bg["dz_w_full"] * bg["rho_w"] * tw
        fz = fz.clone()
        fz[:, :, 0] = 0.0
        fz[:, :, -1] = 0.0
        div_x = op.diff(fx, 0, "u", "m") / bg["dz_m_full"]
        div_y = op.diff(fy, 1, "v", "m") / bg["dz_m_full"]
        div_z = op.diff(fz, 2, "w", "m") * g.dz / bg["dz_m_full"]
        return -bg["C_pi"] * (m_m * (div_x + div_y) + div_z)

    def metric_curvature_tendencies(self, u, v):  # euler.py:188-206
        op, g = self.op, self.grid
        u_m = op.avg(u, 0, "u", "m")
        v_m = op.avg(v, 1, "v", "m")
        v_at_u = op.avg(op.avg(v, 1, "v", "m"), 0, "m", "u")
        u_at_v = op.avg(op.avg(u, 0, "u", "m"), 1, "m", "v")
        metric_m = v_m * g.dm_dx_m[..., None] - u_m * g.dm_dy_m[..., None]
        metric_u = op.avg(metric_m, 0, "m", "u")
        metric_v = op.avg(metric_m, 1, "m", "v")
        return metric_u * v_at_u, -metric_v * u_at_v

    def get_tendencies(self, state_prime, bg, is_explicit=False, ml_params=None):  # euler.py:208-372
        op, g, c = self.op, self.grid, self.c
        u, v, w = state_prime["u"], state_prime["v"], state_prime["w"]
        pi_p, eta = state_prime["pi"], state_prime["eta_dot"]
        if is_explicit:
            th_u = bg["th_v_u"] + state_prime.get("th_v_prime_u", 0.0)
            th_v = bg["th_v_v"] + state_prime.get("th_v_prime_v", 0.0)
            th_w = bg["th_v_w"] + state_prime.get("th_v_prime_w", 0.0)
        else:
            th_u, th_v, th_w = bg["th_v_u"], bg["th_v_v"], bg["th_v_w"]
        gpx = op.diff(pi_p, 0, "m", "u")
        gpy = op.diff(pi_p, 1, "m", "v")
        gpz_w = op.diff(pi_p, 2, "m", "w") * (g.dz / bg["dz_w_full"])
        z_xi_u = op.diff(g.Z_m, 0, "m", "u")
        z_eta_v = op.diff(g.Z_m, 1, "m", "v")
        gpz_m = op.avg(gpz_w, 2, "w", "m")
        gpz_u = op.avg(gpz_m, 0, "m", "u")
        gpz_v = op.avg(gpz_m, 1, "m", "v")
        gx = gpx - z_xi_u * gpz_u
        gy = gpy - z_eta_v * gpz_v
        tend_u = -c["cp"] * th_u * gx
        tend_v = -c["cp"] * th_v * gy
        gpz_w = op.diff(pi_p, 2, "m", "w") * (g.dz / bg["dz_w_full"])
        if is_explicit:
            thp_w = state_prime.get("th_v_prime_w", 0.0)
            buoy = c["g"] * (thp_w / bg["th_v_w"])
            tend_w = -c["cp"] * th_w * gpz_w + buoy
        else:
            tend_w = -c["cp"] * th_w * gpz_w
        v_at_u = op.avg(op.avg(v, 1, "v", "m"), 0, "m", "u")
        u_at_v = op.avg(op.avg(u, 0, "u", "m"), 1, "m", "v")
        tend_u = tend_u + g.f_u[..., None] * v_at_u
        tend_v = tend_v - g.f_v[..., None] * u_at_v
        if is_explicit:
            mu, mv = self.metric_curvature_tendencies(u, v)
            tend_u = tend_u + mu
            tend_v = tend_v + mv
        m_u = g.m_factors["u"][..., None]
        m_v = g.m_factors["v"][..., None]
        m_m = g.m_factors["m"][..., None]
        fx = (u * bg["rho_u"] * bg["th_v_u"] * bg["dz_u"]) / m_u
        fy = (v * bg["rho_v"] * bg["th_v_v"] * bg["dz_v"]) / m_v
        div_x = op.diff(fx, 0, "u", "m") / bg["dz_m_full"]
        div_y = op.diff(fy, 1, "v", "m") / bg["dz_m_full"]
        fz = eta * bg["dz_w_full"] * bg["rho_w"] * bg["th_v_w"]
        fz = torch.cat([torch.zeros_like(fz[:, :, :1]), fz[:, :, 1:-1], torch.zeros_like(fz[:, :, :1])], dim=2)
        div_z = (op.diff(fz, 2, "w", "m") * g.dz) / bg["dz_m_full"]
        tend_pi = -bg["C_pi"] * (m_m * (div_x + div_y) + div_z)
        dth_w = op.diff(bg["th_v"], 2, "m", "w") * (g.dz / bg["dz_w_full"])
        dth_m = op.avg(dth_w, 2, "w", "m")
        w_m = op.avg(w, 2, "w", "m")
        tend_th = -w_m * dth_m
        if is_explicit:
            pdu = pdv = pdw = pdt = 0.0
            if self.nu_h > 0.0 or self.nu_div > 0.0:
                dt_ = self.diffusion.get_tendencies(state_prime, bg_precomputed=bg)
                tend_u = tend_u + dt_.get("u", 0.0)
                tend_v = tend_v + dt_.get("v", 0.0)
                tend_w = tend_w + dt_.get("w", 0.0)
                tend_th = tend_th + dt_.get("th_v", 0.0)
                pdu = pdu + dt_.get("u", 0.0)
                pdv = pdv + dt_.get("v", 0.0)
                pdw = pdw + dt_.get("w", 0.0)
                pdt = pdt + dt_.get("th_v", 0.0)
            if self.physics_suite is not None:
                pt = self.physics_suite.get_explicit_tendencies(
                    state_prime, bg, interior_mask=self.interior_mask, ml_params=ml_params)
                for k in pt:
                    if k == "u":
                        tend_u = tend_u + pt["u"]; pdu = pdu + pt["u"]
                    if k == "v":
                        tend_v = tend_v + pt["v"]; pdv = pdv + pt["v"]
                    if k == "w":
                        tend_w = tend_w + pt["w"]; pdw = pdw + pt["w"]
                    if k == "th_v":
                        tend_th = tend_th + pt["th_v"]; pdt = pdt + pt["th_v"]
            return {"u": tend_u, "v": tend_v, "w": tend_w, "pi": tend_pi, "th_v": tend_th,
                    "phys_diff_u": pdu, "phys_diff_v": pdv, "phys_diff_w": pdw,
                    "phys_diff_th_v": pdt}
        return {"u": tend_u, "v": tend_v, "w": tend_w, "pi": tend_pi, "th_v": tend_th}

    def linear_operator(self, state_prime, bg, dt, alpha=0.55):  # euler.py:374-439
        op, g = self.op, self.grid
        t = self.get_tendencies(state_prime, bg, is_explicit=False)
        u, v, w = state_prime["u"], state_prime["v"], state_prime["w"]
        L_u = u - alpha * dt * t["u"]
        L_v = v - alpha * dt * t["v"]
        L_w = (1.0 + dt * self.tau_damp) * w - alpha * dt * t["w"]
        L_pi = state_prime["pi"] - alpha * dt * t["pi"]
        u_w = op.avg(op.avg(u, 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(v, 1, "v", "m"), 2, "m", "w")
        if 0 in op.periodic_axes:
            L_u = torch.cat([L_u[:-1], L_u[:1]], dim=0)
        else:
            L_u = torch.cat([u[:1], L_u[1:-1], u[-1:]], dim=0)
        if 1 in op.periodic_axes:
            L_v = torch.cat([L_v[:, :-1], L_v[:, :1]], dim=1)
        else:
            L_v = torch.cat([v[:, :1], L_v[:, 1:-1], v[:, -1:]], dim=1)
        m_w = g.m_factors["w"][..., None]
        L_w = torch.cat([w[:, :, :1], L_w[:, :, 1:-1], w[:, :, -1:]], dim=2)
        eta = state_prime["eta_dot"]
        L_eta = alpha * (bg["dz_w_full"] * eta + m_w * (u_w * g.z_xi_w + v_w * g.z_eta_w) - w)
        L_eta = torch.cat([eta[:, :, :1], L_eta[:, :, 1:-1], eta[:, :, -1:]], dim=2)
        return {"u": L_u, "v": L_v, "w": L_w, "pi": L_pi, "eta_dot": L_eta}
