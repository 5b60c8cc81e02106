"""SISL stepper and solvers on the B200 kernels.

Mirrors ``suetes/regional3d/steppers.py``: ``build_dynamical_core``
(:12-88, SISL branch), ``VerticalPreconditioner`` (:125-253),
``SemiLagrangianAdvector3D`` (:256-374), ``SemiImplicitSolver3D``
(:377-527), ``FluxFormAdvector`` (:530-647) and ``SISLStepper3D``
(:650-1073).  Every numerical method calls the C ABI of
``libsisl_b200.so``; a whole step is one ``sisl_step`` call.

Precision follows the state: float32 tensors run the float32 kernels (with
float64 GMRES reductions and Hessenberg algebra), float64 tensors the
float64 kernels.  The thermodynamic fields are carried in perturbation form
(``pi - pi_bg``, ``th_v - theta_bg``) between steps.
"""

import ctypes

import torch

from . import _lib
from ._lib import check, ptrs
from .boundaries import LateralRelaxation
from .core import F64, empty_field, fortran, zeros_field
from .euler import Euler3D

SOLVE_METHODS = {"batched": _lib.SISL_GMRES_BATCHED, "incremental": _lib.SISL_GMRES_INCREMENTAL}
LOC5 = (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("eta_dot", "w"))


def build_dynamical_core(core_type, grid, operators, constants, initial_state, physics_suite=None,
                         interior_mask=None, **kwargs):
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
    params = {"dt": 120.0, "damp_height": 9000.0, "max_damp": 3.0, "nu_div_factor": 0.1, "nu_h_factor": 0.1,
              "N_bv": 0.01, "alpha": 0.55, "use_limiter": False, "use_checkpointing": False,
              "solver_tol": 1e-12, "solver_maxiter": 100, "solver_restart": 100, "background_state": None,
              "solve_method": "batched"}
    params.update(kwargs)
    ref = params["background_state"] if params["background_state"] is not None else initial_state
    physics = Euler3D(grid, operators, constants, dt=params["dt"], initial_era5_state=ref,
                      damp_height=params["damp_height"], max_damp=params["max_damp"],
                      nu_div_factor=params["nu_div_factor"], nu_h_factor=params["nu_h_factor"],
                      N_bv=params["N_bv"], physics_suite=physics_suite, interior_mask=interior_mask)
    if "u_prev" not in initial_state:  # steppers.py:69-80
        initial_state["u_prev"] = initial_state["u"]
        initial_state["v_prev"] = initial_state["v"]
        initial_state["w_prev"] = initial_state["w"]
        initial_state["eta_dot_prev"] = initial_state.get("eta_dot", torch.zeros_like(initial_state["w"]))
        initial_state["tend_th_v_prev"] = torch.zeros_like(initial_state["th_v"])
        initial_state["is_first_step"] = 1.0
        for key in (physics_suite.tracer_keys if physics_suite is not None else []):
            if key in initial_state:
                initial_state[f"tend_{key}_prev"] = torch.zeros_like(initial_state[key])
    stepper = SISLStepper3D(physics, params["dt"], alpha=params["alpha"], use_limiter=params["use_limiter"],
                            use_checkpointing=params["use_checkpointing"], solver_tol=params["solver_tol"],
                            solver_maxiter=params["solver_maxiter"], solver_restart=params["solver_restart"],
                            solve_method=params["solve_method"])
    return stepper, params["dt"]


def _dtype_of(d):
    for v in d.values():
        if torch.is_tensor(v) and v.is_floating_point():
            return v.dtype
    return F64


class VerticalPreconditioner:
    """Column Helmholtz preconditioner M^-1 (steppers.py:125-253)."""

    def __init__(self, physics, dt, alpha=0.55, pi_scale=1000.0):
        if pi_scale != 1000.0:
            raise ValueError("the CUDA preconditioner uses pi_scale = 1000")
        self.physics, self.dt, self.alpha, self.pi_scale = physics, dt, alpha, pi_scale
        self.bg = None

    def precompute_banded(self, bg):
        """The banded factorisation is prepared by the core (sisl_core_create)."""
        self.bg = bg

    def __call__(self, rhs_scaled):
        core = self.physics.core(_dtype_of(rhs_scaled), self.dt, self.alpha, bg=self.physics._bg_arg(self.bg))
        ins = [core.field(rhs_scaled[k], l) for k, l in LOC5]
        outs = [core.new(l) for _, l in LOC5]
        check(core.lib.sisl_precond_apply(core.handle, ptrs(ins, 5), ptrs(outs, 5), core.stream),
              "sisl_precond_apply")
        return {k: o for (k, _), o in zip(LOC5, outs)}

    def transpose(self, cot_scaled):
        """``jax.linear_transpose(M_fn)`` applied to a cotangent (steppers.py:474-476)."""
        core = self.physics.core(_dtype_of(cot_scaled), self.dt, self.alpha, bg=self.physics._bg_arg(self.bg))
        ins = [core.field(cot_scaled[k], l) for k, l in LOC5]
        outs = [core.new(l) for _, l in LOC5]
        check(core.lib.sisl_precond_apply_t(core.handle, ptrs(ins, 5), ptrs(outs, 5), core.stream),
              "sisl_precond_apply_t")
        return {k: o for (k, _), o in zip(LOC5, outs)}


class SemiLagrangianAdvector3D:
    """Trajectories and SL interpolation (steppers.py:256-374)."""

    def __init__(self, grid, physics, dt):
        self.grid, self.physics, self.dt, self.op = grid, physics, dt, physics.op

    def compute_departure_indices(self, state, loc="m", iterations=2):
        """Midpoint departure points in index space (steppers.py:318-360);
        returns a (3, ex, ey, ez) tensor."""
        dtype = _dtype_of({k: state[k] for k in ("u", "v", "eta_dot")})
        core = self.physics.core(dtype, self.dt, 0.55)
        u, v, e = core.field(state["u"], "u"), core.field(state["v"], "v"), core.field(state["eta_dot"], "w")
        ex, ey, ez = core.shape(loc)
        # one (3, ex, ey, ez) tensor whose three slices are x-fastest fields: the
        # kernel writes them in place (no stacking copy)
        out = torch.empty((3, ez, ey, ex), dtype=core.dtype, device=core.device).permute(0, 3, 2, 1)
        co = [out[q] for q in range(3)]
        ws, n = core.workspace(_lib.WS_DEPARTURE)
        check(core.lib.sisl_departure(core.handle, _lib.LOC[loc], u.data_ptr(), v.data_ptr(), e.data_ptr(),
                                      int(iterations), ptrs(co, 3), ws.data_ptr(), n, core.stream),
              "sisl_departure")
        return out

    def advect_linear(self, field, coords):
        from .operators import map_coordinates_linear
        return map_coordinates_linear(field, coords)

    def advect_cubic(self, field, coords, use_limiter=False):
        from .operators import tensor_product_interp_3d
        return tensor_product_interp_3d(field, coords, use_limiter=use_limiter)


class SemiImplicitSolver3D:
    """Preconditioned GMRES Helmholtz solve (steppers.py:377-527)."""

    def __init__(self, physics, dt, alpha=0.55, solver_tol=1e-4, solver_maxiter=20, solver_restart=20,
                 solve_method="batched", refine=True):
        self.physics, self.dt, self.alpha = physics, dt, alpha
        # float32 solves: float64 iterative refinement of the restarted GMRES
        self.refine = bool(refine)
        self.pi_scale = 1000.0
        self.solver_tol, self.solver_maxiter, self.solver_restart = solver_tol, solver_maxiter, solver_restart
        self.solve_method = solve_method
        # transposed (adjoint) solve: tolerance (None: solver_tol, as bwd_solve) and
        # unit-norm scaling of the cotangent (False: the reference's absolute eps floor)
        self.transpose_tol = None
        self.transpose_method = None  # "batched" / "incremental"; None: solve_method
        self.transpose_log = None  # a list collects every transposed solve's statistics
        self.adjoint_normalize = True
        self.last_info = None

    def _core(self, dtype, bg=None):
        core = self.physics.core(dtype, self.dt, self.alpha, bg=self.physics._bg_arg(bg))
        core.set_solver(self.solver_tol, self.solver_maxiter, self.solver_restart, SOLVE_METHODS[self.solve_method])
        core.set_refinement(self.refine)
        return core

    def solve(self, rhs_prime, bg_precomputed, x0=None):
        """Solve A x = b (steppers.py:401-496); x0 None means x0 = rhs.

        Differentiable like ``jax.lax.custom_linear_solve`` (steppers.py:483):
        the cotangent of ``rhs_prime`` is the transpose solve of the
        solution's cotangent; ``x0`` receives none."""
        core = self._core(_dtype_of(rhs_prime), bg_precomputed)
        b = [core.field(rhs_prime[k], l) for k, l in LOC5]
        if torch.is_grad_enabled() and any(t.requires_grad for t in b):
            x = _LinearSolve.apply(self, core, x0, *b)
            return {k: t for (k, _), t in zip(LOC5, x)}
        return {k: t for (k, _), t in zip(LOC5, self._solve_core(core, b, x0))}

    def _solve_core(self, core, b, x0):
        x = [core.new(l) for _, l in LOC5]
        x0p, x0t = None, None
        if x0 is not None:
            x0t = [core.field(x0[k], l).detach() for k, l in LOC5]  # keep alive across the call
            x0p = ctypes.cast(ptrs(x0t, 5), ctypes.c_void_p)
        b = [t.detach() for t in b]
        ws, n = core.workspace(_lib.WS_GMRES)
        info = _lib.SislSolveInfo()
        check(core.lib.sisl_gmres_solve(core.handle, ptrs(b, 5), x0p, ptrs(x, 5), ws.data_ptr(), n, core.stream,
                                        ctypes.byref(info)), "sisl_gmres_solve")
        self.last_info = info.as_dict()
        return x

    def solve_transpose(self, cot_solution, bg_precomputed, dtype=None, x0=None):
        """bwd_solve (steppers.py:473-481): the cotangent of the physical rhs
        from the cotangent of the physical solution; ``x0`` an optional
        initial guess (zero as in the reference otherwise)."""
        core = self._core(dtype or _dtype_of(cot_solution), bg_precomputed)
        g = [core.field(cot_solution[k], l) for k, l in LOC5]
        x0l = [x0[k] for k, _ in LOC5] if x0 is not None else None
        return {k: t for (k, _), t in zip(LOC5, self._solve_transpose_core(core, g, x0l))}

    def _solve_transpose_core(self, core, g, x0=None):
        out = [core.new(l) for _, l in LOC5]
        g = [t.detach() for t in g]
        x0p = None
        if x0 is not None:
            x0 = [core.field(t, l).detach() for t, (_, l) in zip(x0, LOC5)]
            x0p = ctypes.cast(ptrs(x0, 5), ctypes.c_void_p)
        ws, n = core.workspace(_lib.WS_GMRES)
        info = _lib.SislSolveInfo()
        core.set_adjoint(self.transpose_tol, self.adjoint_normalize,
                         None if self.transpose_method is None else SOLVE_METHODS[self.transpose_method])
        check(core.lib.sisl_gmres_solve_transpose(core.handle, ptrs(g, 5), x0p, ptrs(out, 5), ws.data_ptr(), n,
                                                  core.stream, ctypes.byref(info)), "sisl_gmres_solve_transpose")
        self.last_transpose_info = info.as_dict()
        if self.transpose_log is not None:
            self.transpose_log.append(self.last_transpose_info)
        return out

    def matvec_scaled(self, x_scaled, bg_precomputed, transpose=False):
        """A_fn (steppers.py:439-461), or its transpose, on the scaled vector."""
        core = self._core(_dtype_of(x_scaled), bg_precomputed)
        ins = [core.field(x_scaled[k], l) for k, l in LOC5]
        outs = [core.new(l) for _, l in LOC5]
        if transpose:
            ws, n = core.workspace(_lib.WS_OPERATOR)
            check(core.lib.sisl_helmholtz_matvec_t(core.handle, ptrs(ins, 5), ptrs(outs, 5), ws.data_ptr(), n,
                                                   core.stream), "sisl_helmholtz_matvec_t")
        else:
            check(core.lib.sisl_helmholtz_matvec(core.handle, ptrs(ins, 5), ptrs(outs, 5), core.stream),
                  "sisl_helmholtz_matvec")
        return {k: o for (k, _), o in zip(LOC5, outs)}

    def relative_residual(self, solution, rhs_prime, bg_precomputed):
        """``||A x - b|| / ||b||`` in the scaled norm (steppers.py:498-527)."""
        applied = self.physics.linear_operator(solution, bg_precomputed, self.dt, alpha=self.alpha)
        num = torch.zeros((), dtype=F64, device=self.physics.grid.device)
        den = torch.zeros_like(num)
        for k, _ in LOC5:
            s = self.pi_scale if k == "pi" else 1.0
            a = applied[k].double() * s
            r = fortran(rhs_prime[k]).double() * s
            num = num + torch.sum((a - r) ** 2)
            den = den + torch.sum(r ** 2)
        return torch.sqrt(num / torch.clamp(den, min=torch.finfo(F64).tiny))


class _LinearSolve(torch.autograd.Function):
    """custom_linear_solve on the five physical rhs fields: forward GMRES on
    A, backward GMRES on A^T with M^T (steppers.py:463-485)."""

    @staticmethod
    def forward(ctx, solver, core, x0, *b):
        ctx.solver, ctx.core = solver, core
        return tuple(solver._solve_core(core, list(b), x0))

    @staticmethod
    def backward(ctx, *g):
        core = ctx.core
        gs = [zeros_field(core.shape(l), core.dtype, core.device) if t is None else core.field(t, l)
              for t, (_, l) in zip(g, LOC5)]
        return (None, None, None) + tuple(ctx.solver._solve_transpose_core(core, gs))


class FluxFormAdvector:
    """Split flux-form SL mass transport (steppers.py:530-647)."""

    def __init__(self, grid, dt, periodic_axes=(), physics=None):
        self.grid, self.dt, self.periodic_axes, self.physics = grid, dt, frozenset(periodic_axes), physics

    def advect_1d(self, scalar_1d, cfl_inter_1d, periodic=False):
        """advect_1d (steppers.py:552-594) for one line or a batch (..., N)."""
        s = torch.as_tensor(scalar_1d)
        c = torch.as_tensor(cfl_inter_1d).to(device=s.device, dtype=s.dtype)
        N = s.shape[-1]
        sb = s.reshape(-1, N).contiguous()
        cb = c.reshape(-1, N + 1).contiguous()
        out = torch.empty_like(sb)
        lib = _lib.load()
        n = int(lib.sisl_ffsl_lines_workspace_bytes(N, sb.shape[0]))
        ws = torch.empty(max(n, 256), dtype=torch.uint8, device=s.device)
        from .core import DTYPE_CODE, stream_ptr
        check(lib.sisl_ffsl_lines(DTYPE_CODE[s.dtype], N, sb.shape[0], sb.data_ptr(), cb.data_ptr(),
                                  int(bool(periodic)), out.data_ptr(), ws.data_ptr(), n, stream_ptr(s.device)),
              "sisl_ffsl_lines")
        return out.reshape(s.shape)

    def advect_1d_vjp(self, scalar_1d, cfl_inter_1d, out_bar, periodic=False):
        """VJP of ``advect_1d`` (``sisl_ffsl_lines_vjp``): the cotangents of
        the scalar (..., N) and of the interface Courant numbers (..., N + 1)."""
        s = torch.as_tensor(scalar_1d)
        c = torch.as_tensor(cfl_inter_1d).to(device=s.device, dtype=s.dtype)
        N = s.shape[-1]
        sb = s.reshape(-1, N).contiguous()
        cb = c.reshape(-1, N + 1).contiguous()
        ob = torch.as_tensor(out_bar).to(device=s.device, dtype=s.dtype).reshape(-1, N).contiguous()
        gs, gc = torch.empty_like(sb), torch.empty_like(cb)
        lib = _lib.load()
        n = int(lib.sisl_ffsl_lines_vjp_workspace_bytes(N, sb.shape[0]))
        ws = torch.empty(max(n, 256), dtype=torch.uint8, device=s.device)
        from .core import DTYPE_CODE, stream_ptr
        check(lib.sisl_ffsl_lines_vjp(DTYPE_CODE[s.dtype], N, sb.shape[0], sb.data_ptr(), cb.data_ptr(),
                                      int(bool(periodic)), ob.data_ptr(), gs.data_ptr(), gc.data_ptr(),
                                      ws.data_ptr(), n, stream_ptr(s.device)), "sisl_ffsl_lines_vjp")
        return gs.reshape(s.shape), gc.reshape(c.shape)

    def advect_3d_split_vjp(self, field, state, bg_precomputed, out_bar):
        """VJP of ``advect_3d_split`` (``sisl_ffsl_advect_vjp``): cotangents of
        the field and of ``u``, ``v``, ``eta_dot``."""
        if self.physics is None:
            raise RuntimeError("FluxFormAdvector needs the Euler3D physics for its metric coefficients")
        core = self.physics.core(field.dtype, self.dt, 0.55)
        f = core.field(field, "m")
        u, v, e = core.field(state["u"], "u"), core.field(state["v"], "v"), core.field(state["eta_dot"], "w")
        ob = core.field(out_bar, "m")
        gf, gu, gv, ge = core.new("m"), core.new("u"), core.new("v"), core.new("w")
        ws, n = core.workspace(_lib.WS_FFSL_VJP)
        check(core.lib.sisl_ffsl_advect_vjp(core.handle, f.data_ptr(), u.data_ptr(), v.data_ptr(), e.data_ptr(),
                                            ob.data_ptr(), gf.data_ptr(), gu.data_ptr(), gv.data_ptr(), ge.data_ptr(),
                                            ws.data_ptr(), n, core.stream), "sisl_ffsl_advect_vjp")
        return {"field": gf, "u": gu, "v": gv, "eta_dot": ge}

    def advect_3d_split(self, field, state, bg_precomputed):
        if self.physics is None:
            raise RuntimeError("FluxFormAdvector needs the Euler3D physics for its metric coefficients")
        core = self.physics.core(field.dtype, self.dt, 0.55)
        f = core.field(field, "m")
        u, v, e = core.field(state["u"], "u"), core.field(state["v"], "v"), core.field(state["eta_dot"], "w")
        out = core.new("m")
        ws, n = core.workspace(_lib.WS_FFSL)
        check(core.lib.sisl_ffsl_advect(core.handle, f.data_ptr(), u.data_ptr(), v.data_ptr(), e.data_ptr(),
                                        out.data_ptr(), ws.data_ptr(), n, core.stream), "sisl_ffsl_advect")
        return out


class DeviceState:
    """Prognostic state + history on the device, perturbation form."""

    FIELDS = (("u", "u"), ("v", "v"), ("w", "w"), ("eta_dot", "w"), ("pi_p", "m"), ("th_p", "m"), ("rho", "m"),
              ("u_prev", "u"), ("v_prev", "v"), ("w_prev", "w"), ("eta_dot_prev", "w"), ("tend_th_prev", "m"))

    def __init__(self, core, tensors=None, is_first_step=1.0):
        self.core = core
        self.t = {}
        for k, loc in self.FIELDS:
            self.t[k] = tensors[k] if tensors is not None and k in tensors else empty_field(
                core.shape(loc), core.dtype, core.device)
        self.is_first_step = float(is_first_step)

    def c_struct(self):
        s = _lib.SislState()
        for k, _ in self.FIELDS:
            setattr(s, k, self.t[k].data_ptr())
        s.is_first_step = self.is_first_step
        return s


class SISLStepper3D:
    """One SISL timestep (steppers.py:650-1073) as one ``sisl_step`` call."""

    def __init__(self, physics, dt, alpha=0.55, use_limiter=False, use_checkpointing=False, solver_tol=1e-4,
                 solver_maxiter=20, solver_restart=20, solve_method="batched"):
        self.physics, self.dt, self.alpha = physics, dt, alpha
        self.use_limiter = use_limiter
        self.use_checkpointing = use_checkpointing
        self.advector = SemiLagrangianAdvector3D(physics.grid, physics, dt)
        self.ffsl_advector = FluxFormAdvector(physics.grid, dt, periodic_axes=physics.op.periodic_axes,
                                              physics=physics)
        self.implicit_solver = SemiImplicitSolver3D(physics, dt, alpha=alpha, solver_tol=solver_tol,
                                                    solver_maxiter=solver_maxiter, solver_restart=solver_restart,
                                                    solve_method=solve_method)
        suite = physics.physics_suite
        self.tracer_keys = list(suite.tracer_keys) if suite is not None else []
        self.last_info = None

    # ------------------------------------------------------------------
    def core(self, dtype):
        s = self.implicit_solver
        c = self.physics.core(dtype, self.dt, self.alpha, use_limiter=self.use_limiter)
        c.set_solver(s.solver_tol, s.solver_maxiter, s.solver_restart, SOLVE_METHODS[s.solve_method])
        c.set_refinement(s.refine)
        return c

    def to_device_state(self, state, dtype=None):
        """Reference state dict (full pi, th_v) -> DeviceState (perturbations)."""
        cached = state.get("_sisl_state")
        if cached is not None and state.get("pi") is cached[1] and state.get("th_v") is cached[2]:
            return cached[0]
        dtype = dtype or _dtype_of({k: state[k] for k in ("u", "v", "w")})
        core = self.core(dtype)
        ph = self.physics
        f = core.field
        t = {"u": f(state["u"], "u"), "v": f(state["v"], "v"), "w": f(state["w"], "w")}
        eta = state.get("eta_dot")
        t["eta_dot"] = f(eta, "w") if eta is not None else zeros_field(core.shape("w"), dtype, core.device)
        t["pi_p"] = fortran(torch.as_tensor(state["pi"]).to(core.device, F64) - ph.pi_bg, dtype=dtype)
        t["th_p"] = fortran(torch.as_tensor(state["th_v"]).to(core.device, F64) - ph.theta_bg, dtype=dtype)
        t["rho"] = f(state["rho"], "m") if "rho" in state else empty_field(core.shape("m"), dtype, core.device)
        first = float(state.get("is_first_step", 1.0))
        if "u_prev" in state:
            t["u_prev"], t["v_prev"] = f(state["u_prev"], "u"), f(state["v_prev"], "v")
            t["w_prev"], t["eta_dot_prev"] = f(state["w_prev"], "w"), f(state["eta_dot_prev"], "w")
            t["tend_th_prev"] = f(state["tend_th_v_prev"], "m")
        else:
            first = 1.0
            t["u_prev"], t["v_prev"], t["w_prev"], t["eta_dot_prev"] = t["u"], t["v"], t["w"], t["eta_dot"]
            t["tend_th_prev"] = zeros_field(core.shape("m"), dtype, core.device)
        return DeviceState(core, t, first)

    def from_device_state(self, ds):
        ph = self.physics
        t = ds.t
        dt_ = ds.core.dtype
        out = {"u": t["u"], "v": t["v"], "w": t["w"], "eta_dot": t["eta_dot"], "rho": t["rho"],
               "pi": fortran(t["pi_p"].double() + ph.pi_bg, dtype=dt_),
               "th_v": fortran(t["th_p"].double() + ph.theta_bg, dtype=dt_),
               "u_prev": t["u_prev"], "v_prev": t["v_prev"], "w_prev": t["w_prev"],
               "eta_dot_prev": t["eta_dot_prev"], "tend_th_v_prev": t["tend_th_prev"],
               "is_first_step": ds.is_first_step}
        out["_sisl_state"] = (ds, out["pi"], out["th_v"])
        return out

    def step_device(self, ds_in, ds_out, relax=None):
        """Advance ds_in by one step into ds_out (no aliasing between them,
        except ds_out history fields that equal ds_in prognostic fields)."""
        core = ds_in.core
        sin, sout = ds_in.c_struct(), ds_out.c_struct()
        rl = relax.c_struct(core) if relax is not None else None
        ws, n = core.workspace(_lib.WS_STEP)
        info = _lib.SislStepInfo()
        rc = check(core.lib.sisl_step(core.handle, ctypes.byref(sin), ctypes.byref(sout),
                                      ctypes.byref(rl) if rl is not None else None, ws.data_ptr(), n, core.stream,
                                      ctypes.byref(info)), "sisl_step")
        ds_out.is_first_step = 0.0
        self.last_info = {"status": rc, "solves": [info.solve[0].as_dict(), info.solve[1].as_dict()],
                          "kernel_launches": int(info.kernel_launches)}
        return self.last_info

    def _relax_of(self, bc_fn):
        if bc_fn is None or isinstance(bc_fn, LateralRelaxation):
            return bc_fn, None
        return None, bc_fn

    def step(self, state, t, forcing, bc_fn, ml_params=None):
        """SISLStepper3D.step (steppers.py:720-1073).

        With autograd recording and a state field that requires grad, the
        step runs as ``DifferentiableStep`` (differentiable CUDA primitives,
        VJP through the transposed solve) instead of the fused kernel chain."""
        if torch.is_grad_enabled() and any(torch.is_tensor(v) and v.requires_grad for v in state.values()):
            return self._step_differentiable(state, bc_fn)
        if self.physics.physics_suite is not None:
            return self._step_physics(state, forcing, bc_fn, ml_params)
        ds = self.to_device_state(state)
        out = DeviceState(ds.core)
        # history of the new state aliases the old prognostic fields (steppers.py:1061-1064)
        for k in ("u", "v", "w", "eta_dot"):
            out.t[k + "_prev"] = ds.t[k]
        relax, generic = self._relax_of(bc_fn)
        self.step_device(ds, out, relax)
        res = self.from_device_state(out)
        if generic is not None:
            res = self._apply_generic_bc(res, generic, forcing, out)
        return res

    def _ffsl_device(self, core, field, ds):
        """Split flux-form transport of a mass-point field by the winds of
        ``ds`` (steppers.py:863-873), device layout in and out."""
        out = core.new("m")
        ws, n = core.workspace(_lib.WS_FFSL)
        check(core.lib.sisl_ffsl_advect(core.handle, field.data_ptr(), ds.t["u"].data_ptr(), ds.t["v"].data_ptr(),
                                        ds.t["eta_dot"].data_ptr(), out.data_ptr(), ws.data_ptr(), n, core.stream),
              "sisl_ffsl_advect")
        return out

    def _step_physics(self, state, forcing, bc_fn, ml_params):
        """``step`` with a physics suite (steppers.py:720-1073).

        The suite's explicit tendencies of the input state (the state_prime of
        steppers.py:767-784; euler.py:347-366) join the fused CUDA step
        through ``sisl_step_physics``.  Density and the registered tracers
        are carried by flux-form transport with the input winds; the suite's
        state updates, then ``bc_fn``, then the equation of state with the
        tracers' mass kept follow in the reference's order
        (steppers.py:1030-1068)."""
        ph, op, suite = self.physics, self.physics.op, self.physics.physics_suite
        if "rho" not in state:
            raise ValueError("a step with a physics suite needs the density 'rho' in the state")
        ds = self.to_device_state(state)
        core = ds.core
        thp = ds.t["th_p"]
        sp_n = {"u": ds.t["u"], "v": ds.t["v"], "w": ds.t["w"], "th_v": core.field(state["th_v"], "m"),
                "pi": ds.t["pi_p"], "eta_dot": ds.t["eta_dot"], "th_v_prime_u": op.avg(thp, 0, "m", "u"),
                "th_v_prime_v": op.avg(thp, 1, "m", "v"), "th_v_prime_w": op.avg(thp, 2, "m", "w")}
        for k in ("theta_surf", "target_th_v"):
            if k in state:
                sp_n[k] = state[k]
        bg = ph.precompute_bg(ph.bg_state_ref())
        pt = suite.get_explicit_tendencies(sp_n, bg, interior_mask=ph.interior_mask, ml_params=ml_params)
        tend = [core.field(pt[k], loc) if k in pt else None
                for k, loc in (("u", "u"), ("v", "v"), ("w", "w"), ("th_v", "m"))]
        out = DeviceState(core)
        for k in ("u", "v", "w", "eta_dot"):
            out.t[k + "_prev"] = ds.t[k]
        sin, sout = ds.c_struct(), out.c_struct()
        ws, n = core.workspace(_lib.WS_STEP)
        info = _lib.SislStepInfo()
        arr = (ctypes.c_void_p * 4)(*[t.data_ptr() if t is not None else None for t in tend])
        rc = check(core.lib.sisl_step_physics(core.handle, ctypes.byref(sin), ctypes.byref(sout), None, arr, None,
                                              ws.data_ptr(), n, core.stream, ctypes.byref(info)),
                   "sisl_step_physics")
        self.last_info = {"status": rc, "solves": [info.solve[0].as_dict(), info.solve[1].as_dict()],
                          "kernel_launches": int(info.kernel_launches)}
        eps = ph.c.get("eps", 1e-15)
        rho_next = self._ffsl_device(core, ds.t["rho"], ds)
        sn = self.from_device_state(out)
        sn.pop("_sisl_state")
        for k in ("u_prev", "v_prev", "w_prev", "eta_dot_prev", "tend_th_v_prev", "is_first_step"):
            sn.pop(k)
        sn["rho"] = rho_next
        first = float(state.get("is_first_step", 1.0)) == 1.0 or "u_prev" not in state
        for key in self.tracer_keys:
            if key in state:
                q_in = core.field(state[key], "m")
                prev = state.get(f"tend_{key}_prev")
                if not first and prev is not None:  # AB2 of a zero tendency (steppers.py:800-812)
                    q_in = q_in + ph.dt * (-0.5 * core.field(prev, "m"))
                sn[key] = self._ffsl_device(core, ds.t["rho"] * q_in, ds) / (rho_next + eps)
        sn = suite.apply_state_updates(sn)
        relax, generic = self._relax_of(bc_fn)
        if relax is not None:
            sn = relax.apply_state(sn, ph)
        elif generic is not None:
            sn = generic(sn, forcing)
        tmass = {k: sn["rho"] * sn[k] for k in self.tracer_keys if k in sn}
        th_p = fortran(torch.as_tensor(sn["th_v"]).to(core.device, F64) - ph.theta_bg, dtype=core.dtype)
        pi_p = fortran(torch.as_tensor(sn["pi"]).to(core.device, F64) - ph.pi_bg, dtype=core.dtype)
        rho = core.new("m")
        check(core.lib.sisl_eos(core.handle, th_p.data_ptr(), pi_p.data_ptr(), rho.data_ptr(), core.stream),
              "sisl_eos")
        sn["rho"] = rho
        for k, rq in tmass.items():
            sn[k] = rq / (rho + eps)
        sn["u_prev"], sn["v_prev"], sn["w_prev"] = ds.t["u"], ds.t["v"], ds.t["w"]
        sn["eta_dot_prev"] = ds.t["eta_dot"]
        sn["tend_th_v_prev"] = out.t["tend_th_prev"]
        for key in self.tracer_keys:
            if key in sn:
                sn[f"tend_{key}_prev"] = torch.zeros_like(sn[key])
        sn["is_first_step"] = 0.0
        return sn

    def _step_differentiable(self, state, bc_fn):
        from .adjoint import DifferentiableStep
        if self.physics.physics_suite is not None:
            raise NotImplementedError("the differentiable step has no physics-suite cotangents")
        relax, generic = self._relax_of(bc_fn)
        dtype = _dtype_of({k: state[k] for k in ("u", "v", "w")})
        key = ("_dstep", dtype)
        dstep = self.__dict__.get(key)
        if dstep is None:
            dstep = DifferentiableStep(self, dtype)
            self.__dict__[key] = dstep
        core = self.core(dtype)
        f = lambda t, loc: core.field(t, loc)
        ps = {"u": f(state["u"], "u"), "v": f(state["v"], "v"), "w": f(state["w"], "w"),
              "eta_dot": f(state["eta_dot"], "w") if "eta_dot" in state else zeros_field(core.shape("w"), dtype,
                                                                                           core.device),
              "pi_p": state["pi"].to(dtype) - dstep.pi_bg, "th_p": state["th_v"].to(dtype) - dstep.theta_bg}
        first = float(state.get("is_first_step", 1.0))
        if "u_prev" in state:
            for k, loc in (("u_prev", "u"), ("v_prev", "v"), ("w_prev", "w"), ("eta_dot_prev", "w")):
                ps[k] = f(state[k], loc)
        else:
            first = 1.0
        ps["is_first_step"] = first
        out = dstep(ps, relax=relax)
        if generic is not None:  # a user bc_fn, then the equation of state (steppers.py:1036-1058)
            from .adjoint import generic_bc_map
            out = generic_bc_map(self, generic, out)
        return {"u": out["u"], "v": out["v"], "w": out["w"], "eta_dot": out["eta_dot"], "rho": out["rho"],
                "pi": out["pi_p"] + dstep.pi_bg, "th_v": out["th_p"] + dstep.theta_bg,
                "u_prev": state["u"], "v_prev": state["v"], "w_prev": state["w"],
                "eta_dot_prev": ps["eta_dot"], "tend_th_v_prev": out["tend_th_prev"], "is_first_step": 0.0}

    def _apply_generic_bc(self, res, bc_fn, forcing, ds):
        """A user bc_fn runs on the assembled state; the EOS of
        steppers.py:1055-1056 is then recomputed if it changed anything."""
        before = {k: res[k] for k in ("u", "v", "w", "pi", "th_v", "eta_dot")}
        res2 = bc_fn(res, forcing)
        if all(res2.get(k) is before[k] for k in before):
            return res2
        core = ds.core
        ph = self.physics
        f = core.field
        ds.t["u"], ds.t["v"], ds.t["w"] = f(res2["u"], "u"), f(res2["v"], "v"), f(res2["w"], "w")
        ds.t["eta_dot"] = f(res2["eta_dot"], "w")
        ds.t["pi_p"] = fortran(torch.as_tensor(res2["pi"]).to(core.device, F64) - ph.pi_bg, dtype=core.dtype)
        ds.t["th_p"] = fortran(torch.as_tensor(res2["th_v"]).to(core.device, F64) - ph.theta_bg, dtype=core.dtype)
        check(core.lib.sisl_eos(core.handle, ds.t["th_p"].data_ptr(), ds.t["pi_p"].data_ptr(),
                                ds.t["rho"].data_ptr(), core.stream), "sisl_eos")
        out = self.from_device_state(ds)
        for k, v in res2.items():
            if k not in out:
                out[k] = v
        return out

    def integrate(self, state, t_start, num_steps, forcing, bc_fn, graph=True):
        """lax.scan over ``step`` (steppers.py:692-714), device resident.

        With ``graph`` (and at least 4 steps) the steps replay two captured
        CUDA graphs (``PingPong``: every GMRES restart loop decided on the
        device, no host synchronisation inside a step), bitwise the eager
        steps; otherwise one ``sisl_step`` call per step."""
        relax, generic = self._relax_of(bc_fn)
        if generic is not None or self.physics.physics_suite is not None:
            for n in range(num_steps):
                state = self.step(state, t_start + n * self.dt, forcing, bc_fn)
            return state
        cur = self.to_device_state(state)
        if graph and num_steps >= 4:
            pp = PingPong([(self, cur, relax)])
            for _ in range(num_steps - pp.steps_done):
                pp.step()
            if pp.k:
                self.last_info = pp.info(0)
            return self.from_device_state(pp.current()[0])
        ring = StateRing(cur.core)
        for _ in range(num_steps):
            nxt = ring.next_output(cur)
            self.step_device(cur, nxt, relax)
            cur = nxt
        return self.from_device_state(cur)


class StateRing:
    """Three rotating output buffer sets for repeated steps.

    The output of a step may not overlap its input, and the input's history
    fields alias the previous state's prognostic buffers, so the output of
    step n can reuse the buffers of step n - 3."""

    def __init__(self, core):
        self.core = core
        self.sets = [DeviceState(core) for _ in range(3)]
        self.n = 0

    def next_output(self, cur):
        out = self.sets[self.n % 3]
        self.n += 1
        for k in ("u", "v", "w", "eta_dot"):
            out.t[k + "_prev"] = cur.t[k]
        return out


class StepGraph:
    """One step of one or more members as a single CUDA graph (``sisl_step_graph_*``).

    ``members``: sequence of ``(stepper, ds_in, ds_out, relax)``; member m
    advances ``ds_in`` into ``ds_out`` (fixed buffers, distinct cores).  The
    GMRES restart loops are conditional nodes decided on the device, so a
    launch needs no host synchronisation; ``info(m)`` reads the solve
    statistics of the last launch.  ``PingPong`` alternates two graphs for
    repeated steps.

    ``grouped``: each of the step's two solves runs as one GMRES over all
    members, every Krylov phase a single launch over a member/block table
    (``sisl_step_graph_create_grouped``); the members' other work stays
    parallel branches and every member's result is the same bits."""

    def __init__(self, members, tapes=None, grouped=False):
        """``tapes``: optional per-member lists of the ten solve-output
        tensors to record (``sisl_step_graph_create_taped``)."""
        self.lib = _lib.load()
        n = len(members)
        cores, ins, outs, relax, ws, nbytes = [], [], [], [], [], []
        self._keep = []
        for stepper, din, dout, rl in members:
            core = din.core
            if dout.core is not core:
                raise ValueError("input and output states of a member must share a core")
            if core in cores:
                raise ValueError("every member needs its own core")
            cores.append(core)
            ins.append(din.c_struct())
            outs.append(dout.c_struct())
            relax.append(ctypes.pointer(rl.c_struct(core)) if rl is not None else None)
            buf, nb = core.workspace(_lib.WS_STEP)
            ws.append(buf)
            nbytes.append(nb)
            self._keep += [din, dout, rl, buf]
        self.cores = cores
        self.device = cores[0].device
        carr = (ctypes.c_void_p * n)(*[c.handle.value for c in cores])
        iarr = (_lib.SislState * n)(*ins)
        oarr = (_lib.SislState * n)(*outs)
        rarr = (ctypes.c_void_p * n)(*[ctypes.cast(r, ctypes.c_void_p).value if r is not None else None
                                      for r in relax])
        warr = (ctypes.c_void_p * n)(*[b.data_ptr() for b in ws])
        barr = (ctypes.c_size_t * n)(*nbytes)
        self._keep += [carr, iarr, oarr, rarr, warr, barr, relax]
        h = ctypes.c_void_p()
        from .core import stream_ptr
        if grouped:
            tarr = None
            if tapes is not None:
                tarr = (ctypes.c_void_p * (10 * n))(*[t.data_ptr() for tp in tapes for t in tp])
                self._keep += [tarr, tapes]
            check(self.lib.sisl_step_graph_create_grouped(n, carr, iarr, oarr, rarr, tarr, warr, barr,
                                                          stream_ptr(self.device), ctypes.byref(h)),
                  "sisl_step_graph_create_grouped")
        elif tapes is None:
            check(self.lib.sisl_step_graph_create(n, carr, iarr, oarr, rarr, warr, barr, stream_ptr(self.device),
                                                  ctypes.byref(h)), "sisl_step_graph_create")
        else:
            tarr = (ctypes.c_void_p * (10 * n))(*[t.data_ptr() for tp in tapes for t in tp])
            self._keep += [tarr, tapes]
            check(self.lib.sisl_step_graph_create_taped(n, carr, iarr, oarr, rarr, tarr, warr, barr,
                                                        stream_ptr(self.device), ctypes.byref(h)),
                  "sisl_step_graph_create_taped")
        self.handle, self.n = h, n
        self.outs = [m[2] for m in members]

    def launch(self):
        from .core import stream_ptr
        check(self.lib.sisl_step_graph_launch(self.handle, stream_ptr(self.device)), "sisl_step_graph_launch")
        for ds in self.outs:
            ds.is_first_step = 0.0

    def info(self, member=0):
        from .core import stream_ptr
        inf = _lib.SislStepInfo()
        rc = self.lib.sisl_step_graph_info(self.handle, int(member), ctypes.byref(inf), stream_ptr(self.device))
        check(rc, "sisl_step_graph_info")
        return {"status": rc, "solves": [inf.solve[0].as_dict(), inf.solve[1].as_dict()]}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.sisl_step_graph_destroy(h)
            except Exception:
                pass
            self.handle = None


class PingPong:
    """Repeated graph steps of a set of members: two DeviceStates per member
    (A, B) and the graphs A -> B and B -> A; ``step()`` launches the next one.

    The first-step flag (no trajectory extrapolation, steppers.py:748-762)
    is fixed when a graph is captured, so a member still on its first step
    takes that step eagerly here (``steps_done`` counts it)."""

    def __init__(self, members, autotune=False, grouped=False):
        """``members``: sequence of ``(stepper, ds0, relax)``; ds0 is copied.
        ``autotune``: choose each member core's launch shapes (``Core.autotune``)
        before the graphs are captured.  ``grouped``: grouped solves
        (``StepGraph``)."""
        self.a, self.b, spec_ab, spec_ba = [], [], [], []
        self.steps_done = 0
        self.tuning = []
        for stepper, ds0, rl in members:
            core = ds0.core
            if autotune:
                self.tuning.append(core.autotune())
            A, B = DeviceState(core), DeviceState(core)
            if ds0.is_first_step == 1.0:
                stepper.step_device(ds0, A, rl)
                self.steps_done = 1
            else:
                for k, v in ds0.t.items():
                    A.t[k].copy_(v)
            A.is_first_step = B.is_first_step = 0.0
            self.a.append(A)
            self.b.append(B)
            spec_ab.append((stepper, A, B, rl))
            spec_ba.append((stepper, B, A, rl))
        if self.steps_done and any(ds0.is_first_step != 1.0 for _, ds0, _ in members):
            raise ValueError("members must all be on their first step or all past it")
        self.g = [StepGraph(spec_ab, grouped=grouped), StepGraph(spec_ba, grouped=grouped)]
        self.k = 0

    def step(self):
        self.g[self.k % 2].launch()
        self.k += 1

    def current(self):
        return self.b if self.k % 2 == 1 else self.a

    def info(self, member=0):
        return self.g[(self.k - 1) % 2].info(member)
