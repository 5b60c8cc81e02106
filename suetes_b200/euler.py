"""``Euler3D`` with the B200 kernels behind its numerical methods.

Mirrors ``suetes/regional3d/euler.py:13-439``.  The background state
(``theta_bg``, ``pi_bg``, ``tau_damp``; euler.py:56-121) is built once in
float64 on the grid's device.  ``precompute_bg`` returns the reference's
dictionary (for user scripts); the kernels themselves read the coefficient
set that ``sisl_core_create`` derives once per (precision, dt, alpha).
"""

import collections
import ctypes
import math

import torch

from . import _lib
from ._lib import check, ptrs
from .core import F64, Core, fortran

# cores kept per Euler3D for backgrounds other than its own (most recently used)
BG_CORE_CACHE = 4


def jnp_interp(x, xp, fp):
    """``jnp.interp`` with clamped ends (euler.py:82), float64 set-up."""
    n = xp.shape[0]
    i = torch.clamp(torch.searchsorted(xp, x.reshape(-1).contiguous(), right=True), 1, n - 1).reshape(x.shape)
    dxx = xp[i] - xp[i - 1]
    tiny = torch.finfo(F64).eps * 2.0 ** -52
    dx0 = dxx.abs() <= tiny
    f = torch.where(dx0, fp[i - 1], fp[i - 1] + ((x - xp[i - 1]) / torch.where(dx0, torch.ones_like(dxx), dxx))
                    * (fp[i] - fp[i - 1]))
    f = torch.where(x < xp[0], fp[0], f)
    return torch.where(x > xp[-1], fp[-1], f)


class HyperFilter:
    """4th-order terrain-following hyperdiffusion (diffusion.py:80-173) on
    the CUDA kernels: ``get_tendencies`` returns the u, v, w and th_v
    tendencies the explicit kernels add (two Cartesian horizontal Laplacians
    at mass points, staggered back).  It is the filter ``Euler3D`` builds
    (euler.py:124: the physics' ``nu_h``, ``nu_v = 0``); other coefficients
    raise."""

    def __init__(self, grid, operators, nu_h=1e6, nu_v=1e6, physics=None):
        self.grid, self.op, self.nu_h, self.nu_v, self.physics = grid, operators, nu_h, nu_v, physics

    def get_tendencies(self, state_prime, bg_precomputed):
        ph = self.physics
        if ph is None or self.nu_v != 0.0 or self.nu_h != ph.nu_h:
            raise NotImplementedError("the CUDA hyperdiffusion is the filter of an Euler3D (its nu_h, nu_v = 0)")
        g = self.grid
        dtype = ph._dtype_of(state_prime)
        z = lambda loc: torch.zeros(g.shape_of(loc), dtype=dtype, device=g.device)
        sp = {"u": state_prime.get("u", z("u")), "v": state_prime.get("v", z("v")), "w": state_prime.get("w", z("w")),
              "pi": state_prime.get("pi", z("m")), "eta_dot": state_prime.get("eta_dot", z("w"))}
        if "th_v" in state_prime:
            thp = fortran(state_prime["th_v"], dtype=F64) - fortran(bg_precomputed["th_v"], dtype=F64)
        elif "th_v_prime_m" in state_prime:
            thp = state_prime["th_v_prime_m"]
        else:
            thp = z("m")
        _, pd = ph._tendencies(sp, thp.to(dtype), bg_precomputed, True)
        has = {"u": "u" in state_prime, "v": "v" in state_prime, "w": "w" in state_prime,
               "th_v": "th_v" in state_prime or "th_v_prime_m" in state_prime}
        return {k: pd[q] for q, k in enumerate(("u", "v", "w", "th_v")) if has[k]}


class Euler3D:
    """Dry non-hydrostatic Euler core: background state plus operators."""

    def __init__(self, grid, operators, constants, dt, initial_era5_state=None, N_bv=0.01,
                 damp_height=20000.0, max_damp=0.5, nu_div_factor=0.8, nu_h_factor=0.1,
                 physics_suite=None, interior_mask=None):
        self.grid, self.op, self.c, self.dt = grid, operators, dict(constants), float(dt)
        self.nu_div = nu_div_factor * grid.dx ** 2 / (4.0 * dt)   # euler.py:62-67
        self.nu_h = nu_h_factor * grid.dx ** 4 / (64.0 * dt)
        self.physics_suite, self.interior_mask = physics_suite, interior_mask
        g, cp = self.c["g"], self.c["cp"]
        dev = grid.device
        Z_m = grid.Z_m
        if initial_era5_state is not None:  # euler.py:76-85
            z_1d = Z_m.mean(dim=(0, 1))
            th = torch.as_tensor(initial_era5_state["th_v"]).to(device=dev, dtype=F64)
            pi = torch.as_tensor(initial_era5_state["pi"]).to(device=dev, dtype=F64)
            self.theta_bg = jnp_interp(Z_m, z_1d, th.mean(dim=(0, 1)))
            pi_top = pi[:, :, -1].mean()
        else:  # euler.py:86-96
            self.theta_0 = 300.0
            self.theta_bg = (self.theta_0 * torch.exp((N_bv ** 2 / g) * Z_m) if N_bv > 0.0
                             else self.theta_0 * torch.ones_like(Z_m))
            z_max = Z_m.max()
            if N_bv > 0.0:
                pi_top = 1.0 + (g ** 2 / (cp * self.theta_0 * N_bv ** 2)) * (torch.exp(-N_bv ** 2 * z_max / g) - 1.0)
            else:
                pi_top = 1.0 - (g / (cp * self.theta_0)) * z_max
        dz = Z_m[:, :, 1:] - Z_m[:, :, :-1]  # euler.py:100-112
        thw = 0.5 * (self.theta_bg[:, :, 1:] + self.theta_bg[:, :, :-1])
        dpi = -(g * dz) / (cp * thw)
        rev = torch.flip(torch.cumsum(torch.flip(dpi, dims=[-1]), dim=-1), dims=[-1])
        top = torch.full((grid.nx, grid.ny, 1), float(pi_top), dtype=F64, device=dev)
        self.pi_bg = torch.cat([top - rev, top], dim=2)
        zw = grid.Z_w  # euler.py:114-121
        self.tau_damp = torch.where(
            zw > damp_height,
            max_damp * 0.5 * (1.0 + torch.tanh(math.pi * (zw - damp_height) / (grid.Lz - damp_height) - math.pi / 2)),
            torch.zeros_like(zw))
        self._cores = {}  # cores of this physics' own background
        self._bg_cores = collections.OrderedDict()  # other backgrounds, least recently used first
        self.diffusion = HyperFilter(grid, operators, nu_h=self.nu_h, nu_v=0.0, physics=self)  # euler.py:124

    # ------------------------------------------------------------------
    def core(self, dtype, dt=None, alpha=0.55, bg=None, solver=None, use_limiter=False):
        """The CUDA core for a precision, time step, off-centring and background."""
        dt = self.dt if dt is None else float(dt)
        theta, pi = (self.theta_bg, self.pi_bg) if bg is None else (bg["th_v"], bg["pi_bg"])
        rho = None if bg is None else bg.get("rho")
        key = (dtype, dt, float(alpha), id(theta), id(pi), id(rho), bool(use_limiter))
        own = theta is self.theta_bg and pi is self.pi_bg and rho is None
        cache = self._cores if own else self._bg_cores
        hit = cache.get(key)
        if hit is not None:
            if not own:
                cache.move_to_end(key)
            return hit[0]
        core = Core(self.grid, self.c, theta, pi, self.tau_damp, dtype, dt, alpha, self.nu_div, self.nu_h,
                    periodic_axes=self.op.periodic_axes, solver=solver, use_limiter=use_limiter, rho_bg=rho)
        cache[key] = (core, theta, pi, rho)  # keep the background alive while cached
        # a fresh precompute_bg dict per call is a new background: keep only
        # the most recent few of those cores (their coefficients are a
        # full set of 3-D arrays each)
        while not own and len(cache) > BG_CORE_CACHE:
            cache.popitem(last=False)
        return core

    def bg_state_ref(self):
        """Background dict built inside ``step`` (steppers.py:769-774)."""
        c = self.c
        rho = c["p0"] / (c["Rd"] * self.theta_bg) * self.pi_bg ** (c["cvd"] / c["Rd"])
        return {"rho": rho, "pi": self.pi_bg, "th_v": self.theta_bg}

    def precompute_bg(self, bg_state):
        """``precompute_bg`` (euler.py:127-160): face-mapped background
        (float64), the reference's keys.  A density that is not the equation
        of state of ``th_v`` and ``pi`` (to round-off) is also kept under
        ``rho`` for the CUDA core's coefficients; otherwise the core forms
        that density itself."""
        op, g = self.op, self.grid
        th, rho, pi = (torch.as_tensor(bg_state[k]).to(device=g.device, dtype=F64) for k in ("th_v", "rho", "pi"))
        if bg_state.get("th_v") is self.theta_bg and bg_state.get("pi") is self.pi_bg:
            th, pi = self.theta_bg, self.pi_bg
        c = self.c
        eos = c["p0"] / (c["Rd"] * th) * pi ** (c["cvd"] / c["Rd"])
        out = {
            "th_v_u": op.avg(th, 0, "m", "u"), "th_v_v": op.avg(th, 1, "m", "v"), "th_v_w": op.avg(th, 2, "m", "w"),
            "rho_u": op.avg(rho, 0, "m", "u"), "rho_v": op.avg(rho, 1, "m", "v"), "rho_w": op.avg(rho, 2, "m", "w"),
            "dz_m_full": g.dz_m_full, "dz_w_full": g.dz_w_full,
            "dz_u": op.avg(g.dz_m_full, 0, "m", "u"), "dz_v": op.avg(g.dz_m_full, 1, "m", "v"),
            "C_pi": (self.c["Rd"] / self.c["cvd"]) * (pi / (rho * th)), "pi_bg": pi, "th_v": th,
        }
        if not torch.allclose(rho, eos, rtol=1e-13, atol=0.0):
            out["rho"] = rho
        return out

    def _bg_arg(self, bg):
        if bg is None or bg.get("rho") is not None:
            return bg
        if bg.get("th_v") is self.theta_bg and bg.get("pi_bg") is self.pi_bg:
            return None
        if torch.equal(bg["th_v"], self.theta_bg) and torch.equal(bg["pi_bg"], self.pi_bg):
            return None
        return bg

    @staticmethod
    def _dtype_of(d):
        for v in d.values():
            if torch.is_tensor(v) and v.is_floating_point():
                return v.dtype
        return F64

    # ------------------------------------------------------------------
    def linear_operator(self, state_prime, bg, dt, alpha=0.55):
        """Helmholtz operator ``x - alpha dt T_lin(x)`` (euler.py:374-439)."""
        dtype = self._dtype_of(state_prime)
        core = self.core(dtype, dt, alpha, bg=self._bg_arg(bg))
        locs = (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("eta_dot", "w"))
        ins = [core.field(state_prime[k], l) for k, l in locs]
        outs = [core.new(l) for _, l in locs]
        ws, n = core.workspace(_lib.WS_OPERATOR)
        check(core.lib.sisl_linear_operator(core.handle, ptrs(ins, 5), ptrs(outs, 5), ws.data_ptr(), n, core.stream),
              "sisl_linear_operator")
        return {k: o for (k, _), o in zip(locs, outs)}

    def _tendencies(self, state_prime, th_prime, bg, is_explicit):
        dtype = self._dtype_of(state_prime)
        core = self.core(dtype, self.dt, 0.55, bg=self._bg_arg(bg))
        ins = [core.field(state_prime["u"], "u"), core.field(state_prime["v"], "v"),
               core.field(state_prime["w"], "w"), core.field(state_prime["pi"], "m"),
               core.field(state_prime["eta_dot"], "w"), core.field(th_prime, "m")]
        outs = [core.new("u"), core.new("v"), core.new("w"), core.new("m"), core.new("m"), core.new("m")]
        pd = [core.new("u"), core.new("v"), core.new("w"), core.new("m")]
        for t in pd:
            t.zero_()
        pd_arr = ptrs(pd, 4)
        ws, n = core.workspace(_lib.WS_EXPLICIT)
        check(core.lib.sisl_tendencies(core.handle, int(is_explicit), ptrs(ins, 6), ptrs(outs, 6),
                                       ctypes.cast(pd_arr, ctypes.c_void_p), ws.data_ptr(), n, core.stream),
              "sisl_tendencies")
        return outs, pd

    def explicit_tendencies_vjp(self, state_prime, th_prime, bg, tend_bar, phys_diff_bar=None):
        """VJP of the explicit tendencies (``sisl_explicit_tendencies_vjp``).

        ``tend_bar``: cotangents of the tendencies by name (``u``, ``v``,
        ``w``, ``pi`` (linear part), ``th_v``, ``nl_pi`` (nonlinear Exner
        tendency)); ``phys_diff_bar``: of the hyperdiffusion parts (``u``,
        ``v``, ``w``, ``th_v``); missing entries are zero.  Returns the
        cotangents of ``u``, ``v``, ``w``, ``pi``, ``eta_dot`` and ``th_p``
        (the theta perturbation)."""
        dtype = self._dtype_of(state_prime)
        core = self.core(dtype, self.dt, 0.55, bg=self._bg_arg(bg))
        locs = (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("eta_dot", "w"))
        ins = [core.field(state_prime[k], l) for k, l in locs] + [core.field(th_prime, "m")]
        tl = (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("th_v", "m"), ("nl_pi", "m"))
        keep = []

        def arr(d, names, n):
            a = (ctypes.c_void_p * n)()
            for q, (k, l) in enumerate(names):
                if d is not None and d.get(k) is not None:
                    t = core.field(d[k], l)
                    keep.append(t)
                    a[q] = t.data_ptr()
            return a
        tb = arr(tend_bar, tl, 6)
        pb = arr(phys_diff_bar, (("u", "u"), ("v", "v"), ("w", "w"), ("th_v", "m")), 4)
        outs = [core.new(l) for _, l in locs] + [core.new("m")]
        ws, n = core.workspace(_lib.WS_EXPLICIT_VJP)
        check(core.lib.sisl_explicit_tendencies_vjp(core.handle, ptrs(ins, 6), tb, ctypes.cast(pb, ctypes.c_void_p),
                                                    ptrs(outs, 6), ws.data_ptr(), n, core.stream),
              "sisl_explicit_tendencies_vjp")
        return dict(zip(("u", "v", "w", "pi", "eta_dot", "th_p"), outs))

    def get_tendencies(self, state_prime, bg, is_explicit=False, ml_params=None):
        """Tendencies of euler.py:208-372.  The theta perturbation is taken
        from ``state_prime['th_v'] - bg['th_v']`` (or ``th_v_prime_m``); its
        face averages are formed by the kernel."""
        g = self.grid
        if is_explicit:
            if "th_v" in state_prime:
                thp = fortran(state_prime["th_v"], dtype=F64) - fortran(bg["th_v"], dtype=F64)
            elif "th_v_prime_m" in state_prime:
                thp = state_prime["th_v_prime_m"]
            else:
                thp = torch.zeros(g.shape, dtype=F64, device=g.device)
        else:
            thp = torch.zeros(g.shape, dtype=F64, device=g.device)
        thp = thp.to(self._dtype_of(state_prime))
        (tu, tv, tw, tpi, tth, _), pd = self._tendencies(state_prime, thp, bg, is_explicit)
        out = {"u": tu, "v": tv, "w": tw, "pi": tpi, "th_v": tth}
        if is_explicit:
            use = self.nu_h > 0.0 or self.nu_div > 0.0
            out.update({"phys_diff_u": pd[0] if use else 0.0, "phys_diff_v": pd[1] if use else 0.0,
                        "phys_diff_w": pd[2] if use else 0.0, "phys_diff_th_v": pd[3] if use else 0.0})
            if self.physics_suite is not None:  # euler.py:347-366
                pt = self.physics_suite.get_explicit_tendencies(state_prime, bg, interior_mask=self.interior_mask,
                                                                ml_params=ml_params)
                for k in ("u", "v", "w", "th_v"):
                    if k in pt:
                        out[k] = out[k] + pt[k]
                        out["phys_diff_" + k] = out["phys_diff_" + k] + pt[k]
        return out

    def nonlinear_pi_tendency(self, state_prime, th_v_prime, bg):
        """theta'-flux part of Exner continuity (euler.py:162-186)."""
        sp = dict(state_prime)
        sp.setdefault("w", torch.zeros(self.grid.shape_of("w"), dtype=self._dtype_of(state_prime),
                                       device=self.grid.device))
        sp.setdefault("pi", torch.zeros(self.grid.shape, dtype=self._dtype_of(state_prime), device=self.grid.device))
        (_, _, _, _, _, nl), _ = self._tendencies(sp, th_v_prime, bg, True)
        return nl

    def metric_curvature_tendencies(self, u, v):
        """Map-curvature accelerations (metric_u v_at_u, -metric_v u_at_v) at
        the u and v faces (euler.py:188-206), ``sisl_metric_curvature``."""
        dtype = self._dtype_of({"u": u, "v": v})
        core = self.core(dtype, self.dt, 0.55)
        ins = [core.field(u, "u"), core.field(v, "v")]
        outs = [core.new("u"), core.new("v")]
        check(core.lib.sisl_metric_curvature(core.handle, ins[0].data_ptr(), ins[1].data_ptr(), outs[0].data_ptr(),
                                             outs[1].data_ptr(), core.stream), "sisl_metric_curvature")
        return outs[0], outs[1]
