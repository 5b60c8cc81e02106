"""Differentiable SISL step and the checkpointed trajectory VJP.

The reference differentiates ``SISLStepper3D.step`` (steppers.py:720-1073)
with JAX autodiff: departure points are stop-gradiented (steppers.py:764-767),
the implicit solve is a ``custom_linear_solve`` whose transpose is GMRES on
A^T with M^T (steppers.py:463-485), the tricubic VJP scatters the 64 weights,
and the explicit stencils honour the edge-padding ``stop_gradient`` of
``CGridOperator3D`` (operators.py:45-61).  ``DifferentiableStep`` restates
the step as a composition of differentiable CUDA primitives:

* ``CGridOperator3D.diff/avg``: staggered stencil kernels and their
  transposes (``sisl_stagger``);
* ``tensor_product_interp_3d``: tricubic kernel, VJP by ``sisl_tricubic_vjp``;
* the implicit solve: GMRES (``sisl_gmres_solve``), VJP by the transposed
  solve (``sisl_gmres_solve_transpose``), or -- when recomputing a step whose
  solves were recorded by ``sisl_step_taped`` -- the recorded solution;

with pointwise products and sums between them.  ``trajectory_vjp`` runs the
fused forward step (``sisl_step_taped``), keeps each step's input state and
solve outputs (every step, or every ``checkpoint_every`` steps with the
segment recomputed, the chunked ``jax.checkpoint`` of driver.py:102-116), and
sweeps backwards one step at a time through ``DifferentiableStep``.
"""

import ctypes

import torch

from . import _lib
from ._lib import check, ptrs
from .core import F64, empty_field, fortran
from .operators import tensor_product_interp_3d

KEYS5 = ("u", "v", "w", "pi", "eta_dot")
LOCS5 = ("u", "v", "w", "m", "w")
# perturbation-form state: the fields of DeviceState (pi_p = pi - pi_bg, th_p = th_v - theta_bg)
STATE_KEYS = ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho", "u_prev", "v_prev", "w_prev", "eta_dot_prev",
              "tend_th_prev")


class _RecordedSolve(torch.autograd.Function):
    """The implicit solve of a recomputed step: forward returns the solution
    recorded by the fused step, backward is the transposed GMRES solve,
    warm-started from ``warm[slot]`` (the same solve of the step after, in a
    backward sweep) when given, which it then replaces."""

    @staticmethod
    def forward(ctx, solver, core, recorded, warm, slot, *b):
        ctx.solver, ctx.core, ctx.warm, ctx.slot = solver, core, warm, slot
        return tuple(r.clone() for r in recorded)

    @staticmethod
    def backward(ctx, *g):
        core = ctx.core
        gs = [empty_field(core.shape(l), core.dtype, core.device).zero_() if t is None else core.field(t, l)
              for t, l in zip(g, LOCS5)]
        x0 = ctx.warm.get(ctx.slot) if ctx.warm is not None else None
        out = ctx.solver._solve_transpose_core(core, gs, x0)
        if ctx.warm is not None:
            ctx.warm[ctx.slot] = out
        return (None, None, None, None, None) + tuple(out)


class DifferentiableStep:
    """``SISLStepper3D.step`` (steppers.py:720-1073) as differentiable CUDA primitives."""

    def __init__(self, stepper, dtype):
        self.stepper = stepper
        ph = stepper.physics
        self.ph, self.op, self.c = ph, ph.op, ph.c
        g = ph.grid
        self.grid, self.dtype = g, dtype
        self.a, self.dt = float(stepper.alpha), float(stepper.dt)
        op = self.op
        F = lambda t: fortran(t, dtype=dtype, device=g.device)
        self.bg64 = ph.precompute_bg(ph.bg_state_ref())
        self.bg = {k: F(v) for k, v in self.bg64.items()}
        self.theta_bg, self.pi_bg = F(ph.theta_bg), F(ph.pi_bg)
        self.m = {loc: F(g.m_factors[loc])[..., None] for loc in ("m", "u", "v", "w")}
        self.f_u, self.f_v = F(g.f_u)[..., None], F(g.f_v)[..., None]
        self.dmdx, self.dmdy = F(g.dm_dx_m)[..., None], F(g.dm_dy_m)[..., None]
        self.z_xi_w, self.z_eta_w = F(g.z_xi_w), F(g.z_eta_w)
        self.dz = float(g.dz)
        with torch.no_grad():
            b = self.bg64
            z_xi_u = op.diff(g.Z_m, 0, "m", "u")
            z_eta_v = op.diff(g.Z_m, 1, "m", "v")
            self.z_xi_u, self.z_eta_v = F(z_xi_u), F(z_eta_v)
            self.z_xi_m = F(op.avg(z_xi_u, 0, "u", "m"))
            self.z_eta_m = F(op.avg(z_eta_v, 1, "v", "m"))
            self.dzr_w = F(g.dz / b["dz_w_full"])
            dth_w = op.diff(b["th_v"], 2, "m", "w") * (g.dz / b["dz_w_full"])
            self.dth_m = F(op.avg(dth_w, 2, "w", "m"))
            nz = g.nz
            inner = torch.ones(g.shape_of("w"), dtype=F64, device=g.device)
            inner[:, :, 0] = 0.0
            inner[:, :, nz] = 0.0
            self.w_inner = F(inner)
            edge = torch.zeros(g.shape_of("u"), dtype=torch.bool, device=g.device)
            edge[0], edge[-1] = True, True
            self.u_edge = fortran(edge)
            edge = torch.zeros(g.shape_of("v"), dtype=torch.bool, device=g.device)
            edge[:, 0], edge[:, -1] = True, True
            self.v_edge = fortran(edge)
            ground = torch.zeros(g.shape_of("w"), dtype=torch.bool, device=g.device)
            ground[:, :, 0] = True
            self.w_ground = fortran(ground)

    # ---- diffusion.py:93-173 (HyperFilter with nu_v = 0) ----
    def _lap_h(self, f):
        op = self.op
        dfz_m = op.avg(op.diff(f, 2, "m", "w") * self.dzr_w, 2, "w", "m")
        gx = op.diff(f, 0, "m", "u") - self.z_xi_u * op.avg(dfz_m, 0, "m", "u")
        gy = op.diff(f, 1, "m", "v") - self.z_eta_v * op.avg(dfz_m, 1, "m", "v")
        gxm = op.avg(gx, 0, "u", "m")
        div_x = op.diff(gx, 0, "u", "m") - self.z_xi_m * op.avg(op.diff(gxm, 2, "m", "w") * self.dzr_w, 2, "w", "m")
        gym = op.avg(gy, 1, "v", "m")
        div_y = op.diff(gy, 1, "v", "m") - self.z_eta_m * op.avg(op.diff(gym, 2, "m", "w") * self.dzr_w, 2, "w",
                                                                 "m")
        return div_x + div_y

    def _hyper(self, sp, thp):
        op, nu = self.op, self.ph.nu_h
        src = {"u": op.avg(sp["u"], 0, "u", "m"), "v": op.avg(sp["v"], 1, "v", "m"),
               "w": op.avg(sp["w"], 2, "w", "m"), "th_v": thp}
        out = {}
        for k, f in src.items():
            t = -nu * self._lap_h(self._lap_h(f))
            if k == "u":
                out[k] = op.avg(t, 0, "m", "u")
            elif k == "v":
                out[k] = op.avg(t, 1, "m", "v")
            elif k == "w":
                out[k] = op.avg(t, 2, "m", "w")
            else:
                out[k] = t
        return out

    # ---- euler.py:188-206 ----
    def metric_curvature(self, u, v):
        op = self.op
        u_m, v_m = op.avg(u, 0, "u", "m"), op.avg(v, 1, "v", "m")
        metric_m = v_m * self.dmdx - u_m * self.dmdy
        v_at_u = op.avg(v_m, 0, "m", "u")
        u_at_v = op.avg(u_m, 1, "m", "v")
        return op.avg(metric_m, 0, "m", "u") * v_at_u, -op.avg(metric_m, 1, "m", "v") * u_at_v

    # ---- euler.py:162-186 ----
    def nonlinear_pi(self, sp, thp):
        op, bg = self.op, self.bg
        fx = sp["u"] * bg["rho_u"] * op.avg(thp, 0, "m", "u") * bg["dz_u"] / self.m["u"]
        fy = sp["v"] * bg["rho_v"] * op.avg(thp, 1, "m", "v") * bg["dz_v"] / self.m["v"]
        fz = sp["eta_dot"] * bg["dz_w_full"] * bg["rho_w"] * op.avg(thp, 2, "m", "w") * self.w_inner
        div_h = (op.diff(fx, 0, "u", "m") + op.diff(fy, 1, "v", "m")) / bg["dz_m_full"]
        div_z = op.diff(fz, 2, "w", "m") * self.dz / bg["dz_m_full"]
        return -bg["C_pi"] * (self.m["m"] * div_h + div_z)

    # ---- euler.py:208-372, is_explicit=True ----
    def tendencies(self, sp, thp):
        op, bg, c = self.op, self.bg, self.c
        u, v, w, pi_p, eta = sp["u"], sp["v"], sp["w"], sp["pi"], sp["eta_dot"]
        thp_u, thp_v, thp_w = op.avg(thp, 0, "m", "u"), op.avg(thp, 1, "m", "v"), op.avg(thp, 2, "m", "w")
        gpz_w = op.diff(pi_p, 2, "m", "w") * self.dzr_w
        gpz_m = op.avg(gpz_w, 2, "w", "m")
        gx = op.diff(pi_p, 0, "m", "u") - self.z_xi_u * op.avg(gpz_m, 0, "m", "u")
        gy = op.diff(pi_p, 1, "m", "v") - self.z_eta_v * op.avg(gpz_m, 1, "m", "v")
        tend_u = -c["cp"] * (bg["th_v_u"] + thp_u) * gx
        tend_v = -c["cp"] * (bg["th_v_v"] + thp_v) * gy
        tend_w = -c["cp"] * (bg["th_v_w"] + thp_w) * gpz_w + c["g"] * (thp_w / bg["th_v_w"])
        u_m, v_m = op.avg(u, 0, "u", "m"), op.avg(v, 1, "v", "m")
        tend_u = tend_u + self.f_u * op.avg(v_m, 0, "m", "u")
        tend_v = tend_v - self.f_v * op.avg(u_m, 1, "m", "v")
        mu, mv = self.metric_curvature(u, v)
        tend_u, tend_v = tend_u + mu, tend_v + mv
        fx = (u * bg["rho_u"] * bg["th_v_u"] * bg["dz_u"]) / self.m["u"]
        fy = (v * bg["rho_v"] * bg["th_v_v"] * bg["dz_v"]) / self.m["v"]
        fz = eta * bg["dz_w_full"] * bg["rho_w"] * bg["th_v_w"] * self.w_inner
        div_h = (op.diff(fx, 0, "u", "m") + op.diff(fy, 1, "v", "m")) / bg["dz_m_full"]
        div_z = (op.diff(fz, 2, "w", "m") * self.dz) / bg["dz_m_full"]
        tend_pi = -bg["C_pi"] * (self.m["m"] * div_h + div_z)
        tend_th = -op.avg(w, 2, "w", "m") * self.dth_m
        out = {"u": tend_u, "v": tend_v, "w": tend_w, "pi": tend_pi, "th_v": tend_th,
               "phys_diff_u": 0.0, "phys_diff_v": 0.0, "phys_diff_w": 0.0, "phys_diff_th_v": 0.0}
        if self.ph.nu_h > 0.0 or self.ph.nu_div > 0.0:
            h = self._hyper(sp, thp)
            for k in ("u", "v", "w", "th_v"):
                out[k] = out[k] + h[k]
                out["phys_diff_" + k] = h[k]
        return out

    # ---- steppers.py:720-1073 ----
    def departure(self, state):
        """Departure indices of the four staggers (no cotangent, steppers.py:748-767)."""
        adv = self.stepper.advector
        it = int(getattr(self.stepper, "departure_iterations", 2))
        with torch.no_grad():
            first = float(state.get("is_first_step", 1.0)) == 1.0
            tr = {}
            for k in ("u", "v", "eta_dot"):
                x = state[k].detach()
                if "u_prev" in state and not first:
                    x = 1.5 * x - 0.5 * state[k + "_prev"].detach()
                tr[k] = x
            return {loc: adv.compute_departure_indices(tr, loc=loc, iterations=it) for loc in ("u", "v", "w", "m")}

    def __call__(self, state, relax=None, recorded=None, coords=None, warm=None):
        """One step on a perturbation-form state (keys of ``STATE_KEYS`` plus
        ``is_first_step``); returns the next state in the same form.

        ``recorded``: the two five-field solutions of the fused step for this
        state (replaces the forward GMRES solves); ``relax``: a
        ``LateralRelaxation`` bc_fn."""
        op, bg, c, ph = self.op, self.bg, self.c, self.ph
        a, dt = self.a, self.dt
        lim = self.stepper.use_limiter
        cs = coords if coords is not None else self.departure(state)
        thp_n = state["th_p"]
        sp_n = {"u": state["u"], "v": state["v"], "w": state["w"], "pi": state["pi_p"], "eta_dot": state["eta_dot"]}
        tn = self.tendencies(sp_n, thp_n)
        u_in = state["u"] + dt * ((1.0 - a) * tn["u"] + a * tn["phys_diff_u"])
        v_in = state["v"] + dt * ((1.0 - a) * tn["v"] + a * tn["phys_diff_v"])
        w_in = state["w"] + dt * ((1.0 - a) * tn["w"] + a * tn["phys_diff_w"])
        pi_in = sp_n["pi"] + (1.0 - a) * dt * (tn["pi"] + self.nonlinear_pi(sp_n, thp_n))
        th_in = thp_n + (1.0 - a) * dt * tn["th_v"]
        u_w = op.avg(op.avg(state["u"], 0, "u", "m"), 2, "m", "w")
        v_w = op.avg(op.avg(state["v"], 1, "v", "m"), 2, "m", "w")
        res_n = bg["dz_w_full"] * state["eta_dot"] + u_w * self.z_xi_w + v_w * self.z_eta_w - state["w"]
        ac = lambda f, loc: tensor_product_interp_3d(f, cs[loc], use_limiter=lim)
        R_eta = -(1.0 - a) * ac(res_n, "w")
        rhs_u = ac(u_in, "u")
        rhs_v = ac(v_in, "v")
        if 0 in op.periodic_axes:
            rhs_u = torch.cat([rhs_u[:-1], rhs_u[:1]], dim=0)
        else:
            rhs_u = torch.where(self.u_edge, state["u"], rhs_u)
        if 1 in op.periodic_axes:
            rhs_v = torch.cat([rhs_v[:, :-1], rhs_v[:, :1]], dim=1)
        else:
            rhs_v = torch.where(self.v_edge, state["v"], rhs_v)
        rhs_w = ac(w_in, "w")
        rhs_pi = ac(pi_in, "m")
        th_adv = ac(th_in, "m")
        R_eta_adv = R_eta * self.w_inner
        w_m = op.avg(state["w"], 2, "w", "m")
        w_m_next = w_m
        guess = sp_n
        u_g, v_g = rhs_u, rhs_v
        cad = c["cp"] * a * dt
        solver = self.stepper.implicit_solver
        core = solver._core(self.dtype, self.bg64)
        for it in range(2):  # steppers.py:911-998
            t_th = tn["th_v"] + (w_m - w_m_next) * self.dth_m
            thp_next = th_adv + a * dt * t_th
            tpu, tpv, tpw = op.avg(thp_next, 0, "m", "u"), op.avg(thp_next, 1, "m", "v"), op.avg(thp_next, 2, "m", "w")
            buoy = a * dt * (c["g"] * (tpw / bg["th_v_w"]))
            pg = guess["pi"]
            gz_w = op.diff(pg, 2, "m", "w") * self.dzr_w
            gz_m = op.avg(gz_w, 2, "w", "m")
            nl_u = -cad * tpu * (op.diff(pg, 0, "m", "u") - self.z_xi_u * op.avg(gz_m, 0, "m", "u"))
            nl_v = -cad * tpv * (op.diff(pg, 1, "m", "v") - self.z_eta_v * op.avg(gz_m, 1, "m", "v"))
            nl_w = -cad * tpw * gz_w
            nl_div = self.nonlinear_pi(guess, thp_next)
            mu, mv = self.metric_curvature(u_g, v_g)
            rhs_u_k = rhs_u + nl_u + a * dt * mu
            rhs_v_k = rhs_v + nl_v + a * dt * mv
            rhs_pi_k = rhs_pi + a * dt * nl_div
            ugw = op.avg(op.avg(u_g, 0, "u", "m"), 2, "m", "w")
            vgw = op.avg(op.avg(v_g, 1, "v", "m"), 2, "m", "w")
            kb = self.m["w"] * (ugw * self.z_xi_w + vgw * self.z_eta_w)
            rhs_w_k = torch.where(self.w_ground, kb, (rhs_w + buoy + nl_w) * self.w_inner)
            b = [core.field(t, l) for t, l in zip((rhs_u_k, rhs_v_k, rhs_w_k, rhs_pi_k, R_eta_adv), LOCS5)]
            if recorded is not None:
                x = _RecordedSolve.apply(solver, core, recorded[it], warm, it, *b)
            elif torch.is_grad_enabled() and any(t.requires_grad for t in b):
                from .steppers import _LinearSolve
                x = _LinearSolve.apply(solver, core, guess, *b)
            else:
                x = solver._solve_core(core, b, guess)
            nxt = dict(zip(KEYS5, x))
            guess = nxt
            w_m_next = op.avg(nxt["w"], 2, "w", "m")
            u_g, v_g = nxt["u"], nxt["v"]
        u, v = nxt["u"], nxt["v"]
        if ph.nu_div != 0.0:  # steppers.py:1022-1031
            div_h = op.diff(u, 0, "u", "m") + op.diff(v, 1, "v", "m")
            u = u + ph.nu_div * dt * op.diff(div_h, 0, "m", "u")
            v = v + ph.nu_div * dt * op.diff(div_h, 1, "m", "v")
        w, pi_p, th_p = nxt["w"], nxt["pi"], thp_next
        if relax is not None:  # bc_fn blend, then the EOS (steppers.py:1055-1056)
            u, v, w, th_p, pi_p = self._relax(relax, u, v, w, th_p, pi_p)
        rho = c["p0"] / (c["Rd"] * (th_p + self.theta_bg)) * (pi_p + self.pi_bg) ** (c["cvd"] / c["Rd"])
        return {"u": u, "v": v, "w": w, "eta_dot": nxt["eta_dot"], "pi_p": pi_p, "th_p": th_p, "rho": rho,
                "u_prev": state["u"], "v_prev": state["v"], "w_prev": state["w"],
                "eta_dot_prev": state["eta_dot"], "tend_th_prev": tn["th_v"], "is_first_step": 0.0}

    def _relax(self, relax, u, v, w, th_p, pi_p):
        F = lambda t: fortran(torch.as_tensor(t), dtype=self.dtype, device=self.grid.device)
        masks = {"u": F(relax.mask_u)[..., None], "v": F(relax.mask_v)[..., None], "m": F(relax.mask_m)[..., None]}
        vals = {"u": (u, "u"), "v": (v, "v"), "w": (w, "m"), "th_v": (th_p, "m"), "pi": (pi_p, "m")}
        out = {}
        for k, (val, mloc) in vals.items():
            if k in relax.fields:
                ext = relax.exterior.get(k, 0.0)
                ext = F(ext) if torch.is_tensor(ext) else float(ext)
                m = masks[mloc]
                val = (1.0 - m) * val + m * ext
            out[k] = val
        return out["u"], out["v"], out["w"], out["th_v"], out["pi"]


# ---------------------------------------------------------------------------
# trajectory VJP with step checkpointing
# ---------------------------------------------------------------------------
def _taped_step(stepper, ds, relax, record=True):
    """One fused step (``sisl_step_taped``): (next DeviceState, recorded solves or None)."""
    from .steppers import DeviceState
    core = ds.core
    out = DeviceState(core)
    rec = [[core.new(l) for l in LOCS5] for _ in range(2)] if record else None
    tape = ptrs(rec[0] + rec[1], 10) if record else (ctypes.c_void_p * 10)()
    sin, sout = ds.c_struct(), out.c_struct()
    rl = relax.c_struct(core) if relax is not None else None
    ws, n = core.workspace(_lib.WS_STEP)
    info = _lib.SislStepInfo()
    check(core.lib.sisl_step_taped(core.handle, ctypes.byref(sin), ctypes.byref(sout),
                                   ctypes.byref(rl) if rl is not None else None, tape,
                                   ws.data_ptr(), n, core.stream, ctypes.byref(info)), "sisl_step_taped")
    out.is_first_step = 0.0
    stepper.last_info = {"solves": [info.solve[0].as_dict(), info.solve[1].as_dict()]}
    return out, rec


def step_vjp(stepper, state, recorded, cotangents, relax=None):
    """Cotangent of one step's input state (``sisl_step_vjp``): the reverse
    sweep of the fused step in native kernels, the counterpart of
    ``DifferentiableStep`` under autograd.

    ``state``: the step's input ``DeviceState``; ``recorded``: its ten solve
    outputs from ``sisl_step_taped``; ``cotangents``: output-field
    cotangents by ``STATE_KEYS`` name (missing: zero); ``relax``: the
    ``LateralRelaxation`` of the step.  Returns the cotangents of u, v, w,
    eta_dot, pi_p and th_p.  The transposed solves follow the solver's
    ``transpose_tol`` / ``transpose_method`` / ``adjoint_normalize``."""
    core = state.core
    solver = stepper.implicit_solver
    from .steppers import SOLVE_METHODS
    core.set_adjoint(solver.transpose_tol, solver.adjoint_normalize,
                     None if solver.transpose_method is None else SOLVE_METHODS[solver.transpose_method])
    from .steppers import DeviceState
    locs = dict(DeviceState.FIELDS)
    ob = _lib.SislState()
    keep = []
    for k, g in cotangents.items():
        if g is None or k not in locs:
            continue
        g = core.field(g, locs[k])
        keep.append(g)
        setattr(ob, k, g.data_ptr())
    out = {k: core.new(locs[k]) for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p")}
    ib = _lib.SislState()
    for k, t in out.items():
        setattr(ib, k, t.data_ptr())
    sin = state.c_struct()
    rl = relax.c_struct(core) if relax is not None else None
    ws, n = core.workspace(_lib.WS_STEP_VJP)
    info = _lib.SislStepInfo()
    check(core.lib.sisl_step_vjp(core.handle, ctypes.byref(sin), ptrs(recorded[0] + recorded[1], 10),
                                 ctypes.byref(rl) if rl is not None else None, ctypes.byref(ob), ctypes.byref(ib),
                                 ws.data_ptr(), n, core.stream, ctypes.byref(info)), "sisl_step_vjp")
    solver.last_transpose_info = info.solve[1].as_dict()
    if solver.transpose_log is not None:
        solver.transpose_log.extend([info.solve[1].as_dict(), info.solve[0].as_dict()])
    return out


def generic_bc_map(stepper, bc_fn, pre, forcing=None):
    """A user ``bc_fn`` applied to a step's output as the reference applies
    it (steppers.py:1036-1058): the reference state (full ``pi`` and
    ``th_v``, float64) goes through ``bc_fn``, then the equation of state
    re-diagnoses ``rho``.  ``pre``: perturbation-form fields of the step
    output (``DeviceState.t``); returns the post-``bc_fn`` fields in the same
    form and precision.  Differentiable with torch autograd (the history
    fields pass through)."""
    ph = stepper.physics
    c = ph.c
    core_dt = pre["u"].dtype
    res = {"u": pre["u"], "v": pre["v"], "w": pre["w"], "eta_dot": pre["eta_dot"], "rho": pre["rho"],
           "pi": pre["pi_p"].double() + ph.pi_bg, "th_v": pre["th_p"].double() + ph.theta_bg}
    res2 = bc_fn(res, forcing)
    th, pi = res2["th_v"].double(), res2["pi"].double()
    post = dict(pre)
    post.update({"u": res2["u"].to(core_dt), "v": res2["v"].to(core_dt), "w": res2["w"].to(core_dt),
                 "eta_dot": res2["eta_dot"].to(core_dt), "pi_p": (pi - ph.pi_bg).to(core_dt),
                 "th_p": (th - ph.theta_bg).to(core_dt),
                 "rho": (c["p0"] / (c["Rd"] * th) * pi ** (c["cvd"] / c["Rd"])).to(core_dt)})
    return post


def _generic_forward(stepper, bc_fn, pre_ds):
    """The post-``bc_fn`` DeviceState of a fused step's output."""
    from .steppers import DeviceState
    core = pre_ds.core
    locs = dict(DeviceState.FIELDS)
    post = generic_bc_map(stepper, bc_fn, pre_ds.t)
    out = DeviceState(core, {k: core.field(v, locs[k]) for k, v in post.items()}, pre_ds.is_first_step)
    return out


def _generic_cotangents(stepper, bc_fn, pre_ds, g_post):
    """Cotangents of the pre-``bc_fn`` step output from those of the
    post-``bc_fn`` state (autograd through ``generic_bc_map``)."""
    pre = {k: v.detach().requires_grad_(True) for k, v in pre_ds.t.items()}
    with torch.enable_grad():
        post = generic_bc_map(stepper, bc_fn, pre)
        outs, grads = [], []
        for k, g in g_post.items():
            if k in post and post[k].requires_grad:
                outs.append(post[k])
                grads.append(g)
        keys = list(pre)
        gs = torch.autograd.grad(outs, [pre[k] for k in keys], grads, allow_unused=True) if outs else []
    return {k: g for k, g in zip(keys, gs) if g is not None}


def _as_dict(ds):
    d = dict(ds.t)
    d["is_first_step"] = ds.is_first_step
    return d


def trajectory_vjp(stepper, state0, num_steps, objective, bc_fn=None, checkpoint_every=1, wrt=("th_p",),
                   warm_start=False, native=True):
    """Value and gradient of ``J = sum_n objective(n, state_n)`` over
    ``num_steps`` SISL steps from ``state0`` (a reference state dict or a
    ``DeviceState``).

    ``objective(n, state)`` gets the perturbation-form state after step ``n``
    (1-based; keys of ``STATE_KEYS``) and returns a scalar tensor or None.
    Returns ``(J, grads)``, ``grads[k]`` the cotangent of the initial
    ``state[k]`` for ``k`` in ``wrt`` (``th_p`` is the initial theta'; the
    cotangent of th_v is the same).  The forward pass runs the fused step
    and keeps every ``checkpoint_every``-th state; the backward pass
    recomputes a segment with the fused step (recording its solves) and
    differentiates it one step at a time through ``DifferentiableStep``
    (jax.checkpoint of steppers.py:792-850, driver.py:91-132).  With
    ``warm_start`` each transposed solve starts from the same solve's result
    of the step after (the reference's bwd_solve starts from zero; both
    converge to the same cotangent within the solver tolerance).  With
    ``native`` (and no warm start) each step's reverse sweep is one
    ``sisl_step_vjp`` call; otherwise autograd through
    ``DifferentiableStep``.  ``bc_fn``: None, a ``LateralRelaxation`` (fused
    into the step and its sweep) or any torch callable ``bc_fn(state,
    forcing)`` such as ``DaviesSponge.blend`` (``generic_bc_map``: applied
    after the fused step, differentiated with autograd, then the step's
    native sweep)."""
    relax, generic = stepper._relax_of(bc_fn)
    if generic is not None and not native:
        raise NotImplementedError("a user bc_fn is differentiated with the native reverse sweep (native=True)")
    from .steppers import DeviceState
    ds0 = state0 if isinstance(state0, DeviceState) else stepper.to_device_state(state0)
    dstep = DifferentiableStep(stepper, ds0.core.dtype)
    K = max(1, int(checkpoint_every))
    checkpoints = {0: ds0}
    keep_all = K == 1  # every state and solve kept: no recomputation of the forward
    kept_states, kept_recs = [ds0], []
    cur = ds0
    J = torch.zeros((), dtype=F64, device=ds0.core.device)
    pre_states = {}  # step outputs before a generic bc_fn (kept with every state)
    with torch.no_grad():
        for n in range(num_steps):
            cur, rec = _taped_step(stepper, cur, relax, record=keep_all)
            if generic is not None:
                if keep_all:
                    pre_states[n + 1] = cur
                cur = _generic_forward(stepper, generic, cur)
            if keep_all:
                kept_states.append(cur)
                kept_recs.append(rec)
            val = objective(n + 1, _as_dict(cur))
            if val is not None:
                J = J + val.double()
            if (n + 1) % K == 0 and n + 1 < num_steps:
                checkpoints[n + 1] = cur
    keys = [k for k in STATE_KEYS]
    cot = {}
    warm = {} if warm_start else None  # transposed-solve guesses carried along the backward sweep
    for seg0 in range(((num_steps - 1) // K) * K, -1, -K):
        seg1 = min(seg0 + K, num_steps)
        if keep_all:
            states, recs = kept_states[seg0:seg1 + 1], kept_recs[seg0:seg1]
        else:
            states, recs = [checkpoints[seg0]], []
            with torch.no_grad():
                for n in range(seg0, seg1):
                    nxt, rec = _taped_step(stepper, states[-1], relax)
                    if generic is not None:
                        pre_states[n + 1] = nxt
                        nxt = _generic_forward(stepper, generic, nxt)
                    states.append(nxt)
                    recs.append(rec)
        for n in range(seg1 - 1, seg0 - 1, -1):
            after = {k: v.detach().requires_grad_(True) for k, v in states[n + 1 - seg0].t.items()}
            g_after = dict(cot)
            with torch.enable_grad():
                val = objective(n + 1, dict(after, is_first_step=0.0))
                if val is not None and val.requires_grad:
                    gs = torch.autograd.grad(val, [after[k] for k in keys], allow_unused=True)
                    for k, g in zip(keys, gs):
                        if g is not None:
                            g_after[k] = g_after[k] + g if k in g_after else g
            before_ds = states[n - seg0]
            if generic is not None and g_after:
                g_after = _generic_cotangents(stepper, generic, pre_states.pop(n + 1), g_after)
            if native and not warm_start:
                cot = step_vjp(stepper, before_ds, recs[n - seg0], g_after, relax=relax) if g_after else {}
                continue
            before = {k: v.detach().requires_grad_(True) for k, v in before_ds.t.items()}
            with torch.enable_grad():
                out = dstep(dict(before, is_first_step=before_ds.is_first_step), relax=relax,
                            recorded=recs[n - seg0], warm=warm)
                outs, grads = [], []
                for k, g in g_after.items():
                    if k in out and torch.is_tensor(out[k]) and out[k].requires_grad:
                        outs.append(out[k])
                        grads.append(g)
                gs = torch.autograd.grad(outs, [before[k] for k in keys], grads, allow_unused=True) if outs else []
            cot = {k: g for k, g in zip(keys, gs) if g is not None}
    return J, {k: cot.get(k) for k in wrt}


def ensemble_trajectory_vjp(members, num_steps, objective, checkpoint_every=1, wrt=("th_p",), max_workers=None):
    """``trajectory_vjp`` of every member of an ensemble, the members driven
    concurrently: each on its own CUDA stream from its own host thread.  The
    library's calls release the interpreter lock and keep their state in the
    member's core and workspace, so the members' kernels and the
    host round trips of their GMRES restart loops overlap on the GPU.

    ``members``: ``[(stepper, state0, bc_fn)]`` (distinct steppers);
    ``objective(m, n, state)`` as for ``trajectory_vjp`` with the member index
    first.  Returns ``[(J_m, grads_m)]`` in member order, ready on the
    caller's current stream."""
    import concurrent.futures

    from .steppers import DeviceState
    if not members:
        return []
    first = members[0][1]
    dev = torch.device(first.core.device if isinstance(first, DeviceState) else first["u"].device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    base = torch.cuda.current_stream(dev)
    streams = [torch.cuda.Stream(device=dev) for _ in members]

    def run(m):
        torch.cuda.set_device(dev)  # a new host thread starts on device 0
        st, s0, bc = members[m]
        s = streams[m]
        s.wait_stream(base)
        with torch.cuda.stream(s):
            return trajectory_vjp(st, s0, num_steps, lambda n, x: objective(m, n, x), bc_fn=bc,
                                  checkpoint_every=checkpoint_every, wrt=wrt)

    with concurrent.futures.ThreadPoolExecutor(max_workers=max_workers or len(members)) as ex:
        out = list(ex.map(run, range(len(members))))
    for s in streams:
        base.wait_stream(s)
    return out


def _state_struct(fields, is_first_step=0.0):
    """A SislState of the tensors in ``fields`` (STATE_KEYS names; missing: NULL)."""
    s = _lib.SislState()
    for k, t in fields.items():
        if t is not None:
            setattr(s, k, t.data_ptr())
    s.is_first_step = float(is_first_step)
    return s


class StepVJPGraph:
    """The reverse sweep of one step of one or more members as a single CUDA
    graph (``sisl_step_vjp_graph_create``): member m maps the output
    cotangents ``out_bar`` to the input cotangents ``in_bar`` (dicts of
    fixed tensors by ``STATE_KEYS`` name) with its input ``DeviceState`` and
    the ten solve outputs its taped step recorded; the transposed GMRES loops
    are decided on the device.  ``members``: ``(stepper, ds_in, tape, relax,
    out_bar, in_bar)``, distinct cores.  ``grouped``: each transposed solve
    runs as one GMRES over all members, every Krylov phase a single launch
    (``sisl_step_vjp_graph_create_grouped``), with the same bits."""

    def __init__(self, members, grouped=False):
        from .core import stream_ptr
        from .steppers import SOLVE_METHODS
        self.lib = _lib.load()
        n = len(members)
        self._keep = []
        cores, ins, obs, ibs, relax, ws, nbytes, tps = [], [], [], [], [], [], [], []
        for stepper, din, tape, rl, ob, ib in members:
            core = din.core
            if core in cores:
                raise ValueError("every member needs its own core")
            sol = stepper.implicit_solver
            core.set_adjoint(sol.transpose_tol, sol.adjoint_normalize,
                             None if sol.transpose_method is None else SOLVE_METHODS[sol.transpose_method])
            cores.append(core)
            ins.append(din.c_struct())
            obs.append(_state_struct(ob))
            ibs.append(_state_struct(ib))
            relax.append(ctypes.pointer(rl.c_struct(core)) if rl is not None else None)
            buf, nb = core.workspace(_lib.WS_STEP_VJP)
            ws.append(buf)
            nbytes.append(nb)
            tps += [t.data_ptr() for t in tape]
            self._keep += [din, tape, rl, ob, ib, buf]
        self.device = cores[0].device
        carr = (ctypes.c_void_p * n)(*[c.handle.value for c in cores])
        iarr = (_lib.SislState * n)(*ins)
        oarr = (_lib.SislState * n)(*obs)
        barr_ = (_lib.SislState * n)(*ibs)
        tarr = (ctypes.c_void_p * (10 * n))(*tps)
        rarr = (ctypes.c_void_p * n)(*[ctypes.cast(r, ctypes.c_void_p).value if r is not None else None
                                      for r in relax])
        warr = (ctypes.c_void_p * n)(*[b.data_ptr() for b in ws])
        narr = (ctypes.c_size_t * n)(*nbytes)
        self._keep += [carr, iarr, oarr, barr_, tarr, rarr, warr, narr, relax]
        h = ctypes.c_void_p()
        fn = "sisl_step_vjp_graph_create_grouped" if grouped else "sisl_step_vjp_graph_create"
        check(getattr(self.lib, fn)(n, carr, iarr, tarr, rarr, oarr, barr_, warr, narr, stream_ptr(self.device),
                                    ctypes.byref(h)), fn)
        self.handle, self.n = h, n

    def launch(self):
        from .core import stream_ptr
        check(self.lib.sisl_step_graph_launch(self.handle, stream_ptr(self.device)), "sisl_step_graph_launch")

    def info(self, member=0):
        from .core import stream_ptr
        inf = _lib.SislStepInfo()
        rc = self.lib.sisl_step_graph_info(self.handle, int(member), ctypes.byref(inf), stream_ptr(self.device))
        check(rc, "sisl_step_graph_info")
        return {"status": rc, "solves": [inf.solve[1].as_dict(), inf.solve[0].as_dict()]}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.sisl_step_graph_destroy(h)
            except Exception:
                pass
            self.handle = None


class EnsembleVJPGraph:
    """Value and gradient of ``J_m = sum_n objective(m, n, state_m,n)`` over
    ``num_steps`` steps for every member of an ensemble, replayed as CUDA
    graphs: per step one graph advancing every member while recording its
    solves, and one graph of every member's reverse sweep (2 ``num_steps``
    graph launches per evaluation, no host synchronisation inside a step).
    Every state, tape and cotangent buffer is allocated once; ``run`` copies
    the starting states in.  The objective's own cotangents are added
    between the reverse launches (stream-ordered).

    ``members``: ``[(stepper, ds0, relax)]`` with distinct cores; ``ds0``
    fixes the shapes and the first-step flag of every later start.
    ``grouped``: both graphs run their solves grouped over the members
    (``StepGraph``, ``StepVJPGraph``)."""

    def __init__(self, members, num_steps, grouped=False):
        from .steppers import DeviceState, StepGraph
        N = int(num_steps)
        if N < 1:
            raise ValueError("num_steps must be >= 1")
        self.N, self.members = N, members
        self.first = [float(ds0.is_first_step) for _, ds0, _ in members]
        self.S, self.T, self.B = [], [], []
        for stepper, ds0, rl in members:
            core = ds0.core
            S = [DeviceState(core, None, self.first[len(self.S)] if n == 0 else 0.0) for n in range(N + 1)]
            for n in range(N + 1):
                for k in S[n].t:
                    S[n].t[k].zero_()
            T = [[core.new(l) for l in LOCS5 + LOCS5] for _ in range(N)]
            B = [{k: core.new(l).zero_() for k, l in DeviceState.FIELDS} for _ in range(N + 1)]
            self.S.append(S)
            self.T.append(T)
            self.B.append(B)
        M = len(members)
        self.fwd = [StepGraph([(members[m][0], self.S[m][n], self.S[m][n + 1], members[m][2]) for m in range(M)],
                              tapes=[self.T[m][n] for m in range(M)], grouped=grouped) for n in range(N)]
        self.rev = [StepVJPGraph([(members[m][0], self.S[m][n], self.T[m][n], members[m][2], self.B[m][n + 1],
                                   self.B[m][n]) for m in range(M)], grouped=grouped) for n in range(N)]

    def run(self, starts, objective, wrt=("th_p",)):
        """``starts``: a ``DeviceState`` per member (same shapes and first-step
        flag as at construction); ``objective(m, n, state)`` as for
        ``ensemble_trajectory_vjp``.  Returns ``[(J_m, grads_m)]``."""
        M, N = len(self.members), self.N
        for m, ds in enumerate(starts):
            if float(ds.is_first_step) != self.first[m]:
                raise ValueError("a start's first-step flag differs from the captured one")
            for k, t in self.S[m][0].t.items():
                t.copy_(ds.t[k])
        for g in self.fwd:
            g.launch()
        keys = list(STATE_KEYS)
        J = [torch.zeros((), dtype=F64, device=self.S[0][0].core.device) for _ in range(M)]
        G = [[None] * (N + 1) for _ in range(M)]  # objective cotangents per member and state
        for m in range(M):
            for n in range(1, N + 1):
                after = {k: v.detach().requires_grad_(True) for k, v in self.S[m][n].t.items()}
                with torch.enable_grad():
                    val = objective(m, n, dict(after, is_first_step=0.0))
                    if val is None or not val.requires_grad:
                        continue
                    J[m] = J[m] + val.detach().double()
                    gs = torch.autograd.grad(val, [after[k] for k in keys], allow_unused=True)
                G[m][n] = {k: g for k, g in zip(keys, gs) if g is not None}
        for m in range(M):
            for t in self.B[m][N].values():
                t.zero_()
            for k, g in (G[m][N] or {}).items():
                self.B[m][N][k].add_(g)
        for n in range(N - 1, -1, -1):
            if n + 1 < N:  # the reverse of step n + 1 wrote B[n + 1]; add the objective's own cotangent
                for m in range(M):
                    for k, g in (G[m][n + 1] or {}).items():
                        self.B[m][n + 1][k].add_(g)
            self.rev[n].launch()
        return [(J[m], {k: self.B[m][0][k] for k in wrt}) for m in range(M)]
