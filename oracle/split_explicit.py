"""Oracle restatement of the split-explicit RK3 core.

Follows ``suetes/regional3d/steppers.py:1076-1737`` (``SplitExplicitStepper3D``:
three RK3 stages of slow tendencies with 3rd-order upwind flux advection,
each followed by a forward-backward acoustic sub-cycle with a vertically
implicit column solve) and the factory's split branch
(``steppers.py:90-119``).  Float64 torch on the CPU.  Test infrastructure
only: nothing in the product imports it.
"""

import torch

from .linalg import tridiagonal_solve
from .steppers import FluxFormAdvector


class SplitExplicitStepper3D:
    def __init__(self, physics, dt, ns, alpha=0.55):  # steppers.py:1091-1114
        self.physics, self.dt, self.ns, self.alpha = physics, dt, ns, alpha
        self.ns_stage1 = max(1, round(ns / 3))
        self.ns_stage2 = max(1, round(ns / 2))
        self.ns_stage3 = ns
        self.dtau_stage1 = (dt / 3.0) / float(self.ns_stage1)
        self.dtau_stage2 = (dt / 2.0) / float(self.ns_stage2)
        self.dtau_stage3 = dt / float(self.ns_stage3)
        self.ffsl_advector = FluxFormAdvector(physics.grid, dt, periodic_axes=physics.op.periodic_axes)

    def _bg(self):
        ph, c = self.physics, self.physics.c
        rho = c["p0"] / (c["Rd"] * ph.theta_bg) * ph.pi_bg ** (c["cvd"] / c["Rd"])
        return ph.precompute_bg({"rho": rho, "pi": ph.pi_bg, "th_v": ph.theta_bg})

    def _prime(self, s):  # steppers.py:1152-1163, 1381-1393
        ph, op = self.physics, self.physics.op
        thp = s["th_v"] - ph.theta_bg
        sp = {"u": s["u"], "v": s["v"], "w": s["w"], "th_v": s["th_v"], "pi": s["pi"] - ph.pi_bg,
              "eta_dot": s.get("eta_dot", torch.zeros_like(s["w"])),
              "th_v_prime_u": op.avg(thp, 0, "m", "u"), "th_v_prime_v": op.avg(thp, 1, "m", "v"),
              "th_v_prime_w": op.avg(thp, 2, "m", "w")}
        for k in s:
            if k not in sp:
                sp[k] = s[k]
        return sp, thp

    def step(self, state, t, forcing, bc_fn, ml_params=None):  # steppers.py:1117-1270
        ph = self.physics
        bg = self._bg()
        st = state  # the reference diagnoses eta_dot and w into the caller's dict
        st["eta_dot"], st["w"] = self._diagnose_eta_dot(st)
        sp, _ = self._prime(st)
        phys = {}
        diff = {}
        if ph.physics_suite is not None:
            phys = ph.physics_suite.get_explicit_tendencies(sp, bg, interior_mask=ph.interior_mask,
                                                           ml_params=ml_params)
        if ph.nu_h > 0.0 or ph.nu_div > 0.0:
            diff = ph.diffusion.get_tendencies(sp, bg_precomputed=bg)
        suite, nu_h = ph.physics_suite, ph.nu_h
        ph.physics_suite, ph.nu_h = None, 0.0
        try:
            cur = st
            stages = ((self.dtau_stage1, self.ns_stage1), (self.dtau_stage2, self.ns_stage2),
                      (self.dtau_stage3, self.ns_stage3))
            for n, (dtau, ns) in enumerate(stages):
                sf = self._compute_slow_tendencies(cur, bg, phys, diff, ml_params)
                cur = self._acoustic_loop(st, cur, sf, bg, dtau, ns)
                if n < 2:
                    cur["eta_dot"], cur["w"] = self._diagnose_eta_dot(cur)
        finally:
            ph.physics_suite, ph.nu_h = suite, nu_h
        sn = cur
        eps = ph.c.get("eps", 1e-15)
        if suite is not None:
            for key in suite.tracer_keys:
                if key in st:
                    rq = self.ffsl_advector.advect_3d_split(st["rho"] * st[key], st, bg)
                    sn[key] = rq / (sn["rho"] + eps)
        if ph.physics_suite is not None:
            sn = ph.physics_suite.apply_state_updates(sn)
        sn = bc_fn(sn, forcing)
        sn["eta_dot"], sn["w"] = self._diagnose_eta_dot(sn)
        tmass = {}
        if ph.physics_suite is not None:
            tmass = {k: sn["rho"] * sn[k] for k in ph.physics_suite.tracer_keys if k in sn}
        c = ph.c
        sn["rho"] = c["p0"] / (c["Rd"] * sn["th_v"]) * sn["pi"] ** (c["cvd"] / c["Rd"])
        for k, rq in tmass.items():
            sn[k] = rq / (sn["rho"] + eps)
        return sn

    def _diagnose_eta_dot(self, s):  # steppers.py:1272-1310
        ph, op, g = self.physics, self.physics.op, self.physics.grid
        u_w = op.avg(op.avg(s["u"], 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(s["v"], 1, "v", "m"), 2, "m", "w")
        m_w = g.m_factors["w"][..., None]
        w_sfc = m_w[:, :, 0] * (u_w[:, :, 0] * g.z_xi_w[:, :, 0] + v_w[:, :, 0] * g.z_eta_w[:, :, 0])
        w = s["w"].clone()
        w[:, :, 0] = w_sfc
        w[:, :, -1] = 0.0
        ed = (w - m_w * (u_w * g.z_xi_w + v_w * g.z_eta_w)) / g.dz_w_full
        ed[:, :, 0] = 0.0
        ed[:, :, -1] = 0.0
        return ed, w

    def _upwind_flux_3rd_order(self, flux, field, axis):  # steppers.py:1312-1360
        n = field.shape[axis]
        if axis in self.physics.op.periodic_axes:
            idx = torch.arange(-2, n + 2) % n
        else:
            idx = torch.clamp(torch.arange(-2, n + 2), 0, n - 1)
        q = field.index_select(axis, idx)
        qm2 = q.narrow(axis, 0, n + 1)
        qm1 = q.narrow(axis, 1, n + 1)
        q0 = q.narrow(axis, 2, n + 1)
        qp1 = q.narrow(axis, 3, n + 1)
        q4 = (7.0 / 12.0) * (q0 + qm1) - (1.0 / 12.0) * (qp1 + qm2)
        qb = (1.0 / 12.0) * ((qp1 - qm2) - 3.0 * (q0 - qm1))
        clean = torch.where(flux.abs() < self.physics.c.get("eps_l", 1e-12), torch.zeros_like(flux), flux)
        return flux * (q4 + torch.sign(clean) * qb)

    def _compute_slow_tendencies(self, s, bg, phys, diff, ml_params):  # steppers.py:1362-1465
        ph, op, g = self.physics, self.physics.op, self.physics.grid
        sp, thp = self._prime(s)
        tn = ph.get_tendencies(sp, bg, is_explicit=True, ml_params=ml_params)
        tn["pi"] = tn["pi"] + ph.nonlinear_pi_tendency(sp, thp, bg)
        for k in ("u", "v", "w", "th_v"):
            if phys and k in phys:
                tn[k] = tn[k] + phys[k]
            if diff and k in diff:
                tn[k] = tn[k] + diff[k]
        m_m = g.m_factors["m"][..., None]
        m_u = g.m_factors["u"][..., None]
        m_v = g.m_factors["v"][..., None]
        u_m = op.avg(s["u"], 0, "u", "m")
        v_m = op.avg(s["v"], 1, "v", "m")
        w_m = op.avg(s["w"], 2, "w", "m")
        U = sp["u"] / m_u
        V = sp["v"] / m_v
        W = sp["eta_dot"] * bg["dz_w_full"]
        zfac = g.dz / bg["dz_m_full"]
        dU = op.diff(U, 0, "u", "m")
        dV = op.diff(V, 1, "v", "m")
        dW = op.diff(W, 2, "w", "m") * zfac

        def adv(q):
            ax = op.diff(self._upwind_flux_3rd_order(U, q, 0), 0, "u", "m")
            ay = op.diff(self._upwind_flux_3rd_order(V, q, 1), 1, "v", "m")
            az = op.diff(self._upwind_flux_3rd_order(W, q, 2), 2, "w", "m") * zfac
            return -(m_m ** 2) * (ax - q * dU + ay - q * dV) - (az - q * dW)

        tn["th_v"] = tn["th_v"] + adv(thp)
        tn["u"] = tn["u"] + op.avg(adv(u_m), 0, "m", "u")
        tn["v"] = tn["v"] + op.avg(adv(v_m), 1, "m", "v")
        tn["w"] = tn["w"] + op.avg(adv(w_m), 2, "m", "w")
        return tn

    def _acoustic_loop(self, s0, sc, sf, bg, dtau, num_steps):  # steppers.py:1467-1633
        ph, op, g = self.physics, self.physics.op, self.physics.grid
        cp = ph.c["cp"]
        upp = s0["u"] - sc["u"]
        vpp = s0["v"] - sc["v"]
        wpp = s0["w"] - sc["w"]
        ppp = s0["pi"] - sc["pi"]
        m_u = g.m_factors["u"][..., None]
        m_v = g.m_factors["v"][..., None]
        m_m = g.m_factors["m"][..., None]
        z_xi_u = op.diff(g.Z_m, 0, "m", "u")
        z_eta_v = op.diff(g.Z_m, 1, "m", "v")

        def hgrad(p):
            gzw = op.diff(p, 2, "m", "w") * (g.dz / bg["dz_w_full"])
            gzm = op.avg(gzw, 2, "w", "m")
            return (op.diff(p, 0, "m", "u") - z_xi_u * op.avg(gzm, 0, "m", "u"),
                    op.diff(p, 1, "m", "v") - z_eta_v * op.avg(gzm, 1, "m", "v"))

        def divgrad(a, b):
            dv = op.diff(sc["u"] + a, 0, "u", "m") + op.diff(sc["v"] + b, 1, "v", "m")
            return op.diff(dv, 0, "m", "u"), op.diff(dv, 1, "m", "v")

        def edges(a, b):
            ub = s0["u"] - sc["u"]
            vb = s0["v"] - sc["v"]
            a, b = a.clone(), b.clone()
            if 0 in op.periodic_axes:
                a[-1] = a[0]
            else:
                a[0] = ub[0]
                a[-1] = ub[-1]
            if 1 in op.periodic_axes:
                b[:, -1] = b[:, 0]
            else:
                b[:, 0] = vb[:, 0]
                b[:, -1] = vb[:, -1]
            return a, b

        for _ in range(num_steps):
            u_old, v_old, p_old = upp, vpp, ppp
            gx0, gy0 = hgrad(p_old)
            dx0, dy0 = divgrad(u_old, v_old)
            u_h = u_old + 0.5 * dtau * (sf["u"] - cp * bg["th_v_u"] * gx0 + ph.nu_div * dx0)
            v_h = v_old + 0.5 * dtau * (sf["v"] - cp * bg["th_v_v"] * gy0 + ph.nu_div * dy0)
            u_h, v_h = edges(u_h, v_h)
            fx = (u_h * bg["rho_u"] * bg["th_v_u"] * bg["dz_u"]) / m_u
            fy = (v_h * bg["rho_v"] * bg["th_v_v"] * bg["dz_v"]) / m_v
            div_h = m_m * (op.diff(fx, 0, "u", "m") / bg["dz_m_full"] + op.diff(fy, 1, "v", "m") / bg["dz_m_full"])
            ppp, wpp = self._solve_vertical_acoustic_column(ppp, wpp, u_h, v_h, div_h, sf["pi"], sf["w"], bg, dtau)
            gx1, gy1 = hgrad(ppp)
            dxh, dyh = divgrad(u_h, v_h)
            upp = u_old + dtau * (sf["u"] - 0.5 * cp * bg["th_v_u"] * (gx0 + gx1) + ph.nu_div * dxh)
            vpp = v_old + dtau * (sf["v"] - 0.5 * cp * bg["th_v_v"] * (gy0 + gy1) + ph.nu_div * dyh)
            upp, vpp = edges(upp, vpp)
            wt = (sc["w"] + wpp) / (1.0 + dtau * ph.tau_damp)
            wpp = wt - sc["w"]
        out = {"u": sc["u"] + upp, "v": sc["v"] + vpp, "w": sc["w"] + wpp, "pi": sc["pi"] + ppp,
               "th_v": s0["th_v"] + dtau * num_steps * sf["th_v"], "rho": sc["rho"],
               "eta_dot": sc.get("eta_dot", torch.zeros_like(wpp))}
        for k in sc:
            if k not in out:
                out[k] = sc[k]
        return out

    def _solve_vertical_acoustic_column(self, ppp, wpp, upp, vpp, div_h, sf_pi, sf_w, bg,
                                        dtau):  # steppers.py:1635-1737
        ph, op, g = self.physics, self.physics.op, self.physics.grid
        a, cp = self.alpha, ph.c["cp"]
        dz_w, dz_m = bg["dz_w_full"], bg["dz_m_full"]
        u_w = op.avg(op.avg(upp, 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(vpp, 1, "v", "m"), 2, "m", "w")
        m_w = g.m_factors["w"][..., None]
        w_sfc = m_w[:, :, 0] * (u_w[:, :, 0] * g.z_xi_w[:, :, 0] + v_w[:, :, 0] * g.z_eta_w[:, :, 0])
        gnow = op.diff(ppp, 2, "m", "w") * (g.dz / dz_w)
        w_ex = wpp + dtau * (sf_w - cp * bg["th_v_w"] * gnow)
        w_av = (1.0 - a) * wpp + a * w_ex
        w_av[:, :, 0] = w_sfc
        w_av[:, :, -1] = 0.0
        ed = w_av - m_w * (u_w * g.z_xi_w + v_w * g.z_eta_w)
        ed[:, :, 0] = 0.0
        ed[:, :, -1] = 0.0
        fz = ed * bg["rho_w"] * bg["th_v_w"]
        div_z = (op.diff(fz, 2, "w", "m") * g.dz) / dz_m
        dpi_ex = dtau * (sf_pi - bg["C_pi"] * (div_h + div_z))
        gam = (a * dtau) ** 2 * cp * bg["th_v_w"] * bg["rho_w"] * bg["th_v_w"] / dz_w
        gam[:, :, 0] = 0.0
        gam[:, :, -1] = 0.0
        lower = -(bg["C_pi"] / dz_m) * gam[:, :, :-1]
        upper = -(bg["C_pi"] / dz_m) * gam[:, :, 1:]
        main = 1.0 - lower - upper
        dpi = tridiagonal_solve(lower, main, upper, dpi_ex)
        p_next = ppp + dpi
        gd = op.diff(dpi, 2, "m", "w") * (g.dz / dz_w)
        w_next = w_ex - a * dtau * cp * bg["th_v_w"] * gd
        w_next[:, :, 0] = w_sfc
        w_next[:, :, -1] = 0.0
        return p_next, w_next
