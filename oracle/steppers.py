"""Oracle restatement of the SISL stepper and its solvers.

Follows ``suetes/regional3d/steppers.py:12-88`` (factory, SISL branch) and
``:125-1073`` (``VerticalPreconditioner``, ``SemiLagrangianAdvector3D``,
``SemiImplicitSolver3D``, ``FluxFormAdvector``, ``SISLStepper3D``).
Test infrastructure only.
"""

import torch

from . import DTYPE
from .euler import Euler3D
from .linalg import custom_linear_solve, gmres, linear_transpose, tridiagonal_solve
from .ops import map_coordinates_linear, tensor_product_interp_3d

FIELDS5 = ("u", "v", "w", "pi", "eta_dot")


def pack(d):
    return torch.cat([d[k].reshape(-1) for k in FIELDS5])


def unpack(x, like):
    out, o = {}, 0
    for k in FIELDS5:
        n = like[k].numel()
        out[k] = x[o:o + n].reshape(like[k].shape)
        o += n
    return out


def build_dynamical_core(core_type, grid, operators, constants, initial_state,
                         physics_suite=None, interior_mask=None, **kwargs):
    """The factory (steppers.py:12-122): SISL and split-explicit branches."""
    if core_type.lower() == "split-explicit":  # steppers.py:90-119
        from .split_explicit import SplitExplicitStepper3D
        params = {"dt": 40.0, "ns": 3, "damp_height": 12000.0, "max_damp": 3.0, "nu_div_factor": 0.03,
                  "nu_h_factor": 0.03, "N_bv": 0.01, "alpha": 0.55, "background_state": None}
        params.update(kwargs)
        ref = params["background_state"] if params["background_state"] is not None else initial_state
        physics = Euler3D(grid, operators, constants, dt=params["dt"], initial_era5_state=ref,
                          damp_height=params["damp_height"], max_damp=params["max_damp"],
                          nu_div_factor=params["nu_div_factor"], nu_h_factor=params["nu_h_factor"],
                          N_bv=params["N_bv"], physics_suite=physics_suite, interior_mask=interior_mask)
        return SplitExplicitStepper3D(physics, dt=params["dt"], ns=params["ns"], alpha=params["alpha"]), params["dt"]
    if core_type.lower() != "sisl":
        raise ValueError(f"Unknown core_type: '{core_type}'. Use 'sisl' or 'split-explicit'.")
    params = {"dt": 120.0, "damp_height": 9000.0, "max_damp": 3.0, "nu_div_factor": 0.1,
              "nu_h_factor": 0.1, "N_bv": 0.01, "alpha": 0.55, "use_limiter": False,
              "use_checkpointing": False, "solver_tol": 1e-12, "solver_maxiter": 100,
              "solver_restart": 100, "background_state": None}
    params.update(kwargs)
    ref = params["background_state"] if params["background_state"] is not None else initial_state
    physics = Euler3D(grid, operators, constants, dt=params["dt"], initial_era5_state=ref,
                      damp_height=params["damp_height"], max_damp=params["max_damp"],
                      nu_div_factor=params["nu_div_factor"], nu_h_factor=params["nu_h_factor"],
                      N_bv=params["N_bv"], physics_suite=physics_suite,
                      interior_mask=interior_mask)
    if "u_prev" not in initial_state:  # steppers.py:69-80
        initial_state["u_prev"] = initial_state["u"]
        initial_state["v_prev"] = initial_state["v"]
        initial_state["w_prev"] = initial_state["w"]
        initial_state["eta_dot_prev"] = initial_state.get("eta_dot", torch.zeros_like(initial_state["w"]))
        initial_state["tend_th_v_prev"] = torch.zeros_like(initial_state["th_v"])
        initial_state["is_first_step"] = 1.0
        keys = physics_suite.tracer_keys if physics_suite is not None else []
        for key in keys:
            if key in initial_state:
                initial_state[f"tend_{key}_prev"] = torch.zeros_like(initial_state[key])
    stepper = SISLStepper3D(physics, params["dt"], alpha=params["alpha"],
                            use_limiter=params["use_limiter"],
                            use_checkpointing=params["use_checkpointing"],
                            solver_tol=params["solver_tol"], solver_maxiter=params["solver_maxiter"],
                            solver_restart=params["solver_restart"])
    return stepper, params["dt"]


class VerticalPreconditioner:
    """Column Helmholtz preconditioner (steppers.py:125-253)."""

    def __init__(self, physics, dt, alpha=0.55, pi_scale=1000.0):
        self.physics, self.dt, self.alpha, self.pi_scale = physics, dt, alpha, pi_scale

    def precompute_banded(self, bg):  # steppers.py:153-185
        dt, a, cp = self.dt, self.alpha, self.physics.c["cp"]
        self.th_v_w, self.dz_w_full, self.rho_w = bg["th_v_w"], bg["dz_w_full"], bg["rho_w"]
        self.tau_damp = self.physics.tau_damp
        self.K_w = (a * dt * cp * self.th_v_w) / (self.dz_w_full * (1.0 + dt * self.tau_damp))
        P = self.K_w * self.rho_w * self.th_v_w
        P = torch.cat([torch.zeros_like(P[:, :, :1]), P[:, :, 1:-1], torch.zeros_like(P[:, :, :1])], dim=2)
        self.L_pi = (a * dt * bg["C_pi"]) / bg["dz_m_full"]
        self.lower = -self.L_pi * P[:, :, :-1]
        self.upper = -self.L_pi * P[:, :, 1:]
        self.main = 1.0 - self.lower - self.upper

    def __call__(self, r):  # steppers.py:187-253
        ph, op, g = self.physics, self.physics.op, self.physics.grid
        rhs_pi = r["pi"] / self.pi_scale
        rhs_w = r["w"]
        u_w = op.avg(op.avg(r["u"], 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(r["v"], 1, "v", "m"), 2, "m", "w")
        m_w = g.m_factors["w"][..., None]
        kin = m_w * (u_w * g.z_xi_w + v_w * g.z_eta_w)
        wck = rhs_w / (1.0 + self.dt * self.tau_damp) + r["eta_dot"] / self.alpha - kin
        wt = self.rho_w * self.th_v_w * wck
        wt = torch.cat([torch.zeros_like(wt[:, :, :1]), wt[:, :, 1:-1], torch.zeros_like(wt[:, :, :1])], dim=2)
        div = op.diff(wt, 2, "w", "m") * g.dz
        rhs_h = rhs_pi - self.L_pi * div
        pi_p = tridiagonal_solve(self.lower, self.main, self.upper, rhs_h)
        grad = op.diff(pi_p, 2, "m", "w") * (g.dz / self.dz_w_full)
        a, dt, cp = self.alpha, self.dt, ph.c["cp"]
        w_o = (rhs_w - a * dt * cp * self.th_v_w * grad) / (1.0 + dt * self.tau_damp)
        w_o = torch.cat([rhs_w[:, :, :1], w_o[:, :, 1:-1], rhs_w[:, :, -1:]], dim=2)
        eta_o = r["eta_dot"] / self.alpha + w_o - kin
        eta_o = torch.cat([r["eta_dot"][:, :, :1] * self.dz_w_full[:, :, :1], eta_o[:, :, 1:-1],
                           r["eta_dot"][:, :, -1:] * self.dz_w_full[:, :, -1:]], dim=2)
        return {"u": r["u"], "v": r["v"], "w": w_o, "pi": pi_p * self.pi_scale, "eta_dot": eta_o}


class SemiLagrangianAdvector3D:
    """Trajectories and SL interpolation (steppers.py:256-374)."""

    def __init__(self, grid, physics, dt):
        self.grid, self.physics, self.dt, self.op = grid, physics, dt, physics.op

    def _get_index_velocities(self, u, v, eta, loc="m"):  # steppers.py:276-316
        op, g = self.op, self.grid
        if loc == "m":
            ul, vl, wl = op.avg(u, 0, "u", "m"), op.avg(v, 1, "v", "m"), op.avg(eta, 2, "w", "m")
        elif loc == "u":
            ul = u
            vl = op.avg(op.avg(v, 1, "v", "m"), 0, "m", "u")
            wl = op.avg(op.avg(eta, 2, "w", "m"), 0, "m", "u")
        elif loc == "v":
            ul = op.avg(op.avg(u, 0, "u", "m"), 1, "m", "v")
            vl = v
            wl = op.avg(op.avg(eta, 2, "w", "m"), 1, "m", "v")
        elif loc == "w":
            ul = op.avg(op.avg(u, 0, "u", "m"), 2, "m", "w")
            vl = op.avg(op.avg(v, 1, "v", "m"), 2, "m", "w")
            wl = eta
        else:
            raise ValueError(loc)
        mf = g.m_factors[loc][..., None]
        return (ul * mf) / g.dx, (vl * mf) / g.dy, wl

    def compute_departure_indices(self, state, loc="m", iterations=2):  # steppers.py:318-360
        ui, vi, wi = self._get_index_velocities(state["u"], state["v"], state["eta_dot"], loc)
        g = self.grid
        ex = g.nx + (1 if loc == "u" else 0)
        ey = g.ny + (1 if loc == "v" else 0)
        ez = g.nz + (1 if loc == "w" else 0)
        X, Y, Z = torch.meshgrid(torch.arange(ex, dtype=DTYPE), torch.arange(ey, dtype=DTYPE),
                                 torch.arange(ez, dtype=DTYPE), indexing="ij")
        ax, ay, az = self.dt * ui, self.dt * vi, self.dt * wi
        for _ in range(iterations):
            mid = (X - 0.5 * ax, Y - 0.5 * ay, Z - 0.5 * az)
            ax = self.dt * self.advect_linear(ui, mid)
            ay = self.dt * self.advect_linear(vi, mid)
            az = self.dt * self.advect_linear(wi, mid)
        return torch.stack([X - ax, Y - ay, Z - az], dim=0)

    def advect_linear(self, field, coords):  # steppers.py:362-367
        return map_coordinates_linear(field, coords)

    def advect_cubic(self, field, coords, use_limiter=False):  # steppers.py:369-374
        return tensor_product_interp_3d(field, coords, use_limiter=use_limiter)


class SemiImplicitSolver3D:
    """GMRES Helmholtz solve with its transpose (steppers.py:377-527)."""

    def __init__(self, physics, dt, alpha=0.55, solver_tol=1e-4, solver_maxiter=20,
                 solver_restart=20, solve_method="batched"):
        self.physics, self.dt, self.alpha = physics, dt, alpha
        self.pi_scale = 1000.0
        self.solver_tol, self.solver_maxiter, self.solver_restart = solver_tol, solver_maxiter, solver_restart
        self.solve_method = solve_method
        self.last_stats = {}

    def solve(self, rhs_prime, bg, x0=None):  # steppers.py:401-496
        ps = self.pi_scale
        rhs_s = {k: rhs_prime[k] * ps if k == "pi" else rhs_prime[k] for k in FIELDS5}
        if x0 is not None:
            x0_s = {"u": x0["u"], "v": x0["v"], "w": x0["w"], "pi": x0["pi"] * ps,
                    "eta_dot": x0["eta_dot"] * bg["dz_w_full"]}
        else:
            x0_s = rhs_s
        pre = VerticalPreconditioner(self.physics, self.dt, alpha=self.alpha, pi_scale=ps)
        pre.precompute_banded(bg)
        like = rhs_s

        def M_fn(x):
            return pack(pre(unpack(x, like)))

        op = self.physics.op

        def A_fn(x):
            s = unpack(x, like)
            sp = {"u": s["u"], "v": s["v"], "w": s["w"], "pi": s["pi"] / ps,
                  "eta_dot": s["eta_dot"] / bg["dz_w_full"]}
            old = op.use_stop_grad
            op.use_stop_grad = False
            try:
                L = self.physics.linear_operator(sp, bg, self.dt, alpha=self.alpha)
            finally:
                op.use_stop_grad = old
            return pack({"u": L["u"], "v": L["v"], "w": L["w"], "pi": L["pi"] * ps,
                         "eta_dot": L["eta_dot"]})

        b = pack(rhs_s)
        x0f = pack(x0_s).detach()
        n = b.numel()
        stats = {}

        def fwd_solve(bb):
            return gmres(A_fn, bb, x0=x0f, tol=self.solver_tol, maxiter=self.solver_maxiter,
                         restart=self.solver_restart, M=M_fn, solve_method=self.solve_method,
                         stats=stats)

        def bwd_solve(gg):
            A_T = linear_transpose(A_fn, n)
            M_T = linear_transpose(M_fn, n)
            st = {}
            y = gmres(A_T, gg, x0=None, tol=self.solver_tol, maxiter=self.solver_maxiter,
                      restart=self.solver_restart, M=M_T, solve_method=self.solve_method, stats=st)
            self.last_stats["transpose"] = st
            return y

        xs = custom_linear_solve(b, fwd_solve, bwd_solve)
        self.last_stats["forward"] = stats
        s = unpack(xs, like)
        return {"u": s["u"], "v": s["v"], "w": s["w"], "pi": s["pi"] / ps,
                "eta_dot": s["eta_dot"] / bg["dz_w_full"]}

    def relative_residual(self, solution, rhs_prime, bg):  # steppers.py:498-527
        applied = self.physics.linear_operator(solution, bg, self.dt, alpha=self.alpha)
        ps = self.pi_scale
        num = 0.0
        den = 0.0
        for k in FIELDS5:
            a = applied[k] * ps if k == "pi" else applied[k]
            r = rhs_prime[k] * ps if k == "pi" else rhs_prime[k]
            num = num + torch.sum((a - r) ** 2)
            den = den + torch.sum(r ** 2)
        tiny = torch.finfo(DTYPE).tiny
        return torch.sqrt(num / torch.clamp(den, min=tiny))


class FluxFormAdvector:
    """Directionally split FFSL mass transport (steppers.py:530-647)."""

    def __init__(self, grid, dt, periodic_axes=()):
        self.grid, self.dt, self.periodic_axes = grid, dt, frozenset(periodic_axes)

    def advect_1d(self, scalar_1d, cfl_inter_1d, periodic=False):  # steppers.py:552-594
        return self._advect_last(scalar_1d[None], cfl_inter_1d[None], periodic)[0]

    def _advect_last(self, s, cfl, periodic):
        """advect_1d batched over leading axes (the line axis is last)."""
        N = s.shape[-1]
        if periodic:
            ext = torch.cat([s, s, s], dim=-1)
            M = torch.nn.functional.pad(torch.cumsum(ext, dim=-1), (1, 0))
            idx = torch.arange(N + 1, dtype=s.dtype) + N
            dep = idx - cfl
        else:
            M = torch.nn.functional.pad(torch.cumsum(s, dim=-1), (1, 0))
            idx = torch.arange(N + 1, dtype=s.dtype)
            # jnp.clip is maximum then minimum: at an exact tie each passes half
            # the cotangent (torch.clamp would pass all of it)
            lo_b = torch.zeros((), dtype=s.dtype)
            hi_b = torch.full((), float(N), dtype=s.dtype)
            dep = torch.minimum(torch.maximum(idx - cfl, lo_b), hi_b)
        L = M.shape[-1]
        lo = torch.floor(dep)
        w = dep - lo
        lo = lo.to(torch.int64)
        i0 = torch.clamp(lo, 0, L - 1)
        i1 = torch.clamp(lo + 1, 0, L - 1)
        Md = (1.0 - w) * torch.gather(M, -1, i0) + w * torch.gather(M, -1, i1)
        return Md[..., 1:] - Md[..., :-1]

    def advect_3d_split(self, field, state, bg):  # steppers.py:596-647
        g = self.grid
        m_u = g.m_factors["u"][..., None]
        m_v = g.m_factors["v"][..., None]
        cfl_x = (state["u"] * m_u * self.dt) / g.dx
        cfl_y = (state["v"] * m_v * self.dt) / g.dy
        cfl_z = state["eta_dot"] * self.dt
        m_sq = g.m_factors["m"][..., None] ** 2
        vol = (g.dx * g.dy / m_sq) * bg["dz_m_full"]
        mass = field * vol
        mx = self._advect_last(mass.permute(1, 2, 0), cfl_x.permute(1, 2, 0),
                               0 in self.periodic_axes).permute(2, 0, 1)
        my = self._advect_last(mx.permute(0, 2, 1), cfl_y.permute(0, 2, 1),
                               1 in self.periodic_axes).permute(0, 2, 1)
        mz = self._advect_last(my, cfl_z, False)
        return mz / vol


class SISLStepper3D:
    """One SISL timestep (steppers.py:650-1073)."""

    def __init__(self, physics, dt, alpha=0.55, use_limiter=False, use_checkpointing=False,
                 solver_tol=1e-4, solver_maxiter=20, solver_restart=20, solve_method="batched"):
        self.physics, self.dt, self.alpha = physics, dt, alpha
        self.use_limiter = use_limiter
        self.advector = SemiLagrangianAdvector3D(physics.grid, physics, dt)
        self.ffsl_advector = FluxFormAdvector(physics.grid, dt, periodic_axes=physics.op.periodic_axes)
        self.implicit_solver = SemiImplicitSolver3D(physics, dt, alpha=alpha, solver_tol=solver_tol,
                                                    solver_maxiter=solver_maxiter,
                                                    solver_restart=solver_restart,
                                                    solve_method=solve_method)
        self.use_checkpointing = use_checkpointing
        self.tracer_keys = physics.physics_suite.tracer_keys if physics.physics_suite is not None else []
        self.solve_stats = []
        # The reference stop-gradients the departure points (steppers.py:764-767);
        # True differentiates through them instead (a test switch: with it and
        # CGridOperator3D.use_stop_grad = False the gradient is the exact
        # derivative of the discrete step)
        self.departure_gradient = False

    def integrate(self, state, t_start, num_steps, forcing, bc_fn):  # steppers.py:692-714
        for n in range(num_steps):
            state = self.step(state, t_start + n * self.dt, forcing, bc_fn)
        return state

    def step(self, state, t, forcing, bc_fn, ml_params=None):  # steppers.py:720-1073
        ph, op, g, c = self.physics, self.physics.op, self.physics.grid, self.physics.c
        a, dt = self.alpha, self.dt
        state = dict(state)
        if "eta_dot" not in state:
            state["eta_dot"] = torch.zeros_like(state["w"])
        is_first = float(state.get("is_first_step", 1.0))
        if "u_prev" in state:
            ex = lambda k: state[k] if is_first == 1.0 else 1.5 * state[k] - 0.5 * state[k + "_prev"]
            traj = {"u": ex("u"), "v": ex("v"), "w": ex("w"), "eta_dot": ex("eta_dot")}
        else:
            traj = state
        with torch.set_grad_enabled(self.departure_gradient and torch.is_grad_enabled()):
            tr = {k: (traj[k] if self.departure_gradient else traj[k].detach()) for k in ("u", "v", "eta_dot")}
            cu = self.advector.compute_departure_indices(tr, loc="u")
            cv = self.advector.compute_departure_indices(tr, loc="v")
            cw = self.advector.compute_departure_indices(tr, loc="w")
            cm = self.advector.compute_departure_indices(tr, loc="m")
        bg = ph.precompute_bg(ph.bg_state_ref())
        thp_n = state["th_v"] - ph.theta_bg
        sp_n = {"u": state["u"], "v": state["v"], "w": state["w"], "th_v": state["th_v"],
                "pi": state["pi"] - ph.pi_bg, "eta_dot": state["eta_dot"],
                "th_v_prime_u": op.avg(thp_n, 0, "m", "u"),
                "th_v_prime_v": op.avg(thp_n, 1, "m", "v"),
                "th_v_prime_w": op.avg(thp_n, 2, "m", "w")}
        if "theta_surf" in state:
            sp_n["theta_surf"] = state["theta_surf"]
        if "target_th_v" in state:
            sp_n["target_th_v"] = state["target_th_v"]
        tn = ph.get_tendencies(sp_n, bg, True, ml_params)
        u_in = state["u"] + dt * ((1.0 - a) * tn["u"] + a * tn.get("phys_diff_u", 0.0))
        v_in = state["v"] + dt * ((1.0 - a) * tn["v"] + a * tn.get("phys_diff_v", 0.0))
        w_in = state["w"] + dt * ((1.0 - a) * tn["w"] + a * tn.get("phys_diff_w", 0.0))
        nl_pi_n = ph.nonlinear_pi_tendency(sp_n, thp_n, bg)
        pi_in = sp_n["pi"] + (1.0 - a) * dt * (tn["pi"] + nl_pi_n)
        th_in = thp_n + (1.0 - a) * dt * tn["th_v"]
        tracers_in = {}
        for key in self.tracer_keys:
            if key in state:
                tr_in = state[key]
                if "u_prev" in state:
                    ext = 1.5 * tn.get(key, 0.0) - 0.5 * state.get(f"tend_{key}_prev", 0.0)
                    eff = tn.get(key, 0.0) if is_first == 1.0 else ext
                else:
                    eff = tn.get(key, 0.0)
                tracers_in[key] = tr_in + dt * eff
        u_w = op.avg(op.avg(state["u"], 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(state["v"], 1, "v", "m"), 2, "m", "w")
        res_n = bg["dz_w_full"] * state["eta_dot"] + u_w * g.z_xi_w + v_w * g.z_eta_w - state["w"]
        ac = self.advector.advect_cubic
        R_eta = -(1.0 - a) * ac(res_n, cw, self.use_limiter)
        rhs_u = ac(u_in, cu, self.use_limiter)
        rhs_v = ac(v_in, cv, self.use_limiter)
        if 0 in op.periodic_axes:
            rhs_u = torch.cat([rhs_u[:-1], rhs_u[:1]], dim=0)
        else:
            rhs_u = torch.cat([state["u"][:1], rhs_u[1:-1], state["u"][-1:]], dim=0)
        if 1 in op.periodic_axes:
            rhs_v = torch.cat([rhs_v[:, :-1], rhs_v[:, :1]], dim=1)
        else:
            rhs_v = torch.cat([state["v"][:, :1], rhs_v[:, 1:-1], state["v"][:, -1:]], dim=1)
        rhs_w = ac(w_in, cw, self.use_limiter)
        rhs_pi = ac(pi_in, cm, self.use_limiter)
        th_adv = ac(th_in, cm, self.use_limiter)
        th_v_next = th_adv + a * dt * tn["th_v"] + ph.theta_bg
        rho_next = self.ffsl_advector.advect_3d_split(state["rho"], state, bg)
        tracers_next = {}
        for key in self.tracer_keys:
            if key in state:
                rq = self.ffsl_advector.advect_3d_split(state["rho"] * tracers_in[key], state, bg)
                tracers_next[key] = rq / (rho_next + c.get("eps", 1e-15))
        z = torch.zeros_like(R_eta[:, :, :1])
        R_eta_adv = torch.cat([z, R_eta[:, :, 1:-1], z], dim=2)
        dth_w = op.diff(bg["th_v"], 2, "m", "w") * (g.dz / bg["dz_w_full"])
        dth_m = op.avg(dth_w, 2, "w", "m")
        w_m = op.avg(state["w"], 2, "w", "m")
        m_w = g.m_factors["w"][..., None]
        w_m_next = w_m
        guess = sp_n
        u_g, v_g = rhs_u, rhs_v
        z_xi_u = op.diff(g.Z_m, 0, "m", "u")
        z_eta_v = op.diff(g.Z_m, 1, "m", "v")
        self.solve_stats = []
        for _ in range(2):  # steppers.py:911-998
            t_th = tn["th_v"] + (w_m - w_m_next) * dth_m
            th_v_next = th_adv + a * dt * t_th + ph.theta_bg
            thp_next = th_v_next - ph.theta_bg
            tpu = op.avg(thp_next, 0, "m", "u")
            tpv = op.avg(thp_next, 1, "m", "v")
            tpw = op.avg(thp_next, 2, "m", "w")
            buoy = a * dt * (c["g"] * (tpw / bg["th_v_w"]))
            pg = guess["pi"]
            gx = op.diff(pg, 0, "m", "u")
            gy = op.diff(pg, 1, "m", "v")
            gz_w = op.diff(pg, 2, "m", "w") * (g.dz / bg["dz_w_full"])
            gz_m = op.avg(gz_w, 2, "w", "m")
            gz_u = op.avg(gz_m, 0, "m", "u")
            gz_v = op.avg(gz_m, 1, "m", "v")
            cad = c["cp"] * a * dt
            nl_u = -cad * tpu * (gx - z_xi_u * gz_u)
            nl_v = -cad * tpv * (gy - z_eta_v * gz_v)
            nl_w = -cad * tpw * gz_w
            nl_div = ph.nonlinear_pi_tendency(guess, thp_next, bg)
            mu, mv = ph.metric_curvature_tendencies(u_g, v_g)
            rhs_u_k = rhs_u + nl_u + a * dt * mu
            rhs_v_k = rhs_v + nl_v + a * dt * mv
            rhs_w_k = rhs_w + buoy + nl_w
            rhs_pi_k = rhs_pi + a * dt * nl_div
            ugw = op.avg(op.avg(u_g, 0, "u", "m"), 2, "m", "w")
            vgw = op.avg(op.avg(v_g, 1, "v", "m"), 2, "m", "w")
            kb = m_w[:, :, 0] * (ugw[:, :, 0] * g.z_xi_w[:, :, 0] + vgw[:, :, 0] * g.z_eta_w[:, :, 0])
            rhs_w_k = torch.cat([kb[..., None], rhs_w_k[:, :, 1:-1], torch.zeros_like(kb[..., None])], dim=2)
            rhs_k = {"u": rhs_u_k, "v": rhs_v_k, "w": rhs_w_k, "pi": rhs_pi_k, "eta_dot": R_eta_adv}
            nxt = self.implicit_solver.solve(rhs_k, bg, x0=guess)
            self.solve_stats.append(dict(self.implicit_solver.last_stats.get("forward", {})))
            guess = nxt
            w_m_next = op.avg(nxt["w"], 2, "w", "m")
            u_g, v_g = nxt["u"], nxt["v"]
        sn = {"u": nxt["u"], "v": nxt["v"], "w": nxt["w"], "pi": nxt["pi"] + ph.pi_bg,
              "rho": rho_next, "th_v": th_v_next, "eta_dot": nxt["eta_dot"]}
        for key in self.tracer_keys:
            if key in tracers_next:
                sn[key] = tracers_next[key]
        div_h = op.diff(sn["u"], 0, "u", "m") + op.diff(sn["v"], 1, "v", "m")
        sn["u"] = sn["u"] + ph.nu_div * dt * op.diff(div_h, 0, "m", "u")
        sn["v"] = sn["v"] + ph.nu_div * dt * op.diff(div_h, 1, "m", "v")
        if ph.physics_suite is not None:
            sn = ph.physics_suite.apply_state_updates(sn)
        sn = bc_fn(sn, forcing)
        tmass = {k: sn["rho"] * sn[k] for k in self.tracer_keys if k in sn}
        cvd, Rd, p0 = c["cvd"], c["Rd"], c["p0"]
        sn["rho"] = p0 / (Rd * sn["th_v"]) * sn["pi"] ** (cvd / Rd)
        for k, rq in tmass.items():
            sn[k] = rq / (sn["rho"] + c.get("eps", 1e-15))
        sn["u_prev"], sn["v_prev"], sn["w_prev"] = state["u"], state["v"], state["w"]
        sn["eta_dot_prev"] = state["eta_dot"]
        sn["tend_th_v_prev"] = tn["th_v"]
        for key in self.tracer_keys:
            sn[f"tend_{key}_prev"] = tn.get(key, torch.zeros_like(sn[key]))
        sn["is_first_step"] = 0.0
        return sn
