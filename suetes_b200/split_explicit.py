"""``SplitExplicitStepper3D`` on the B200 kernels.

Mirrors ``suetes/regional3d/steppers.py:1076-1737``: a WRF-style RK3 step
whose three stages each evaluate the slow tendencies (explicit dynamics,
3rd-order upwind flux advection, the physics and hyperdiffusion
tendencies of the step start) and advance the fast acoustic modes with a
forward-backward horizontal / vertically implicit sub-cycle.  The stages
run in one ``sisl_split_step`` call; the physics suite, the tracer
transport (``sisl_ffsl_advect``), ``bc_fn``, the final eta_dot diagnosis
(``sisl_split_diagnose``) and the equation of state (``sisl_eos``) follow
on the host side in the reference's order (steppers.py:1233-1270).
"""

import ctypes

import torch

from . import _lib
from ._lib import check
from .boundaries import LateralRelaxation
from .core import F64, fortran

LOCS4 = (("u", "u"), ("v", "v"), ("w", "w"), ("th_v", "m"))


class SplitExplicitStepper3D:
    """Split-explicit RK3 core (steppers.py:1076-1114 for the constructor)."""

    def __init__(self, physics, dt, ns, alpha=0.55):
        from .steppers import FluxFormAdvector
        self.physics, self.dt, self.ns, self.alpha = physics, dt, ns, alpha
        self.ns_stage1 = max(1, round(ns / 3))
        self.ns_stage2 = max(1, round(ns / 2))
        self.ns_stage3 = ns
        self.dtau_stage1 = (dt / 3.0) / float(self.ns_stage1)
        self.dtau_stage2 = (dt / 2.0) / float(self.ns_stage2)
        self.dtau_stage3 = dt / float(self.ns_stage3)
        self.ffsl_advector = FluxFormAdvector(physics.grid, dt, periodic_axes=physics.op.periodic_axes,
                                              physics=physics)
        self._tau = {}

    def core(self, dtype):
        return self.physics.core(dtype, self.dt, self.alpha)

    def _tau_damp(self, core):
        key = (core.dtype, str(core.device))
        if key not in self._tau:
            self._tau[key] = core.field(self.physics.tau_damp, "w")
        return self._tau[key]

    def _diagnose(self, core, u, v, w):
        """``_diagnose_eta_dot`` (steppers.py:1272-1310): (eta_dot, w)."""
        eta, w_out = core.new("w"), core.new("w")
        check(core.lib.sisl_split_diagnose(core.handle, u.data_ptr(), v.data_ptr(), w.data_ptr(), eta.data_ptr(),
                                           w_out.data_ptr(), core.stream), "sisl_split_diagnose")
        return eta, w_out

    def _eos(self, core, th_v, pi):
        ph = self.physics
        th_p = fortran(torch.as_tensor(th_v).to(core.device, F64) - ph.theta_bg, dtype=core.dtype)
        pi_p = fortran(torch.as_tensor(pi).to(core.device, F64) - ph.pi_bg, dtype=core.dtype)
        rho = core.new("m")
        check(core.lib.sisl_eos(core.handle, th_p.data_ptr(), pi_p.data_ptr(), rho.data_ptr(), core.stream),
              "sisl_eos")
        return rho

    def step_device(self, core, st, phys=None):
        """The three RK3 stages from a diagnosed device state ``st`` (dict of
        u, v, w, eta_dot, pi_p, th_p, rho in the core's layout) into a new
        dict of the same fields (rho copied through)."""
        from .steppers import DeviceState
        ds_in = DeviceState(core, st)
        ds_out = DeviceState(core)
        sin, sout = ds_in.c_struct(), ds_out.c_struct()
        arr = (ctypes.c_void_p * 4)()  # all null: no physics tendencies
        if phys is not None:
            arr = (ctypes.c_void_p * 4)(*[t.data_ptr() if t is not None else None for t in phys])
        ws, n = core.workspace(_lib.WS_SPLIT)
        eps_l = float(self.physics.c.get("eps_l", 1e-12))
        check(core.lib.sisl_split_step(core.handle, ctypes.byref(sin), ctypes.byref(sout), int(self.ns),
                                       float(self.alpha), eps_l, self._tau_damp(core).data_ptr(), arr,
                                       ws.data_ptr(), n, core.stream), "sisl_split_step")
        return {k: ds_out.t[k] for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho")}

    def step_vjp_device(self, core, st, out_bar, deterministic=True):
        """Cotangents of ``step_device``'s input fields (u, v, w, eta_dot,
        pi_p, th_p of the diagnosed state ``st``) from those of its output
        (``out_bar``: dict of the same names, missing entries zero) through
        ``sisl_split_step_vjp``: the three RK3 stages differentiated as XLA
        differentiates the reference's (no physics tendencies).
        ``deterministic``: fixed-point scatters (the same bits on every run)
        or float atomic adds (faster, order-dependent last bits)."""
        from .steppers import DeviceState
        ds_in = DeviceState(core, st)
        ob = DeviceState(core, {k: out_bar[k] for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p") if k in out_bar})
        ib = DeviceState(core)
        sin, sob, sib = ds_in.c_struct(), ob.c_struct(), ib.c_struct()
        for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p"):
            if k not in out_bar:
                setattr(sob, k, None)
        ws, n = core.workspace(_lib.WS_SPLIT_VJP)
        eps_l = float(self.physics.c.get("eps_l", 1e-12))
        check(core.lib.sisl_split_step_vjp(core.handle, ctypes.byref(sin), ctypes.byref(sob), ctypes.byref(sib),
                                           int(self.ns), float(self.alpha), eps_l, self._tau_damp(core).data_ptr(),
                                           int(bool(deterministic)), ws.data_ptr(), n, core.stream),
              "sisl_split_step_vjp")
        return {k: ib.t[k] for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p")}

    def step_vjp(self, state, cot, bc_fn=None, forcing=None):
        """``step`` (without a physics suite) and the cotangents of its input
        state, as ``jax.vjp`` of SplitExplicitStepper3D.step
        (steppers.py:1117-1270) gives them.  ``cot``: cotangents of the
        output's u, v, w, eta_dot, pi, th_v, rho (missing keys zero).
        Returns ``(new_state, grads)`` with grads for u, v, w, eta_dot, pi,
        th_v, rho of the input (the input's eta_dot and rho are overwritten
        by the step's diagnosis and equation of state: zero).

        Native reverse pieces: the output diagnosis^T and the input
        diagnosis^T (``sisl_split_diagnose_vjp``), the three stages^T
        (``sisl_split_step_vjp``); the equation of state's derivative
        (rho/th_v and rho cvd/(Rd pi), elementwise) and a torch ``bc_fn``
        (autograd) are applied in between on the device."""
        ph = self.physics
        if ph.physics_suite is not None:
            raise NotImplementedError("the split-explicit VJP covers the core without a physics suite")
        dtype = state["u"].dtype if torch.is_tensor(state["u"]) else F64
        core = self.core(dtype)
        f = core.field
        din = self.device_state(core, state)
        res = self.step_device(core, din)
        pi = fortran(res["pi_p"].double() + ph.pi_bg, dtype=dtype)
        th = fortran(res["th_p"].double() + ph.theta_bg, dtype=dtype)
        pre = {"u": res["u"], "v": res["v"], "w": res["w"], "eta_dot": res["eta_dot"], "pi": pi, "th_v": th,
               "rho": din["rho"]}
        # bc_fn on the stage output, recorded for its cotangents
        if bc_fn is not None:
            leaves = {k: t.detach().clone().requires_grad_(True) for k, t in pre.items()}
            with torch.enable_grad():
                post = bc_fn(dict(leaves), forcing)
            post_d = {k: (post[k].detach() if torch.is_tensor(post[k]) else post[k]) for k in pre}
        else:
            leaves, post, post_d = None, None, dict(pre)
        u1, v1 = f(post_d["u"], "u"), f(post_d["v"], "v")
        eta2, w2 = self._diagnose(core, u1, v1, f(post_d["w"], "w"))
        rho2 = self._eos(core, post_d["th_v"], post_d["pi"])
        out = dict(state)
        out.pop("_sisl_state", None)
        out.update({"u": u1, "v": v1, "w": w2, "eta_dot": eta2, "pi": f(post_d["pi"], "m"),
                    "th_v": f(post_d["th_v"], "m"), "rho": rho2})
        locs = {"u": "u", "v": "v", "w": "w", "eta_dot": "w", "pi": "m", "th_v": "m", "rho": "m"}

        def cz(k):
            t = cot.get(k)
            return f(t, locs[k]).clone() if t is not None else torch.zeros_like(f(pre[k], locs[k]))

        # equation of state: rho = p0 / (Rd th_v) pi^(cvd/Rd)
        c = ph.c
        rb = cz("rho")
        g = {k: cz(k) for k in ("u", "v", "pi", "th_v")}
        g["th_v"] = g["th_v"] - rb * rho2 / out["th_v"]
        g["pi"] = g["pi"] + rb * rho2 * (c["cvd"] / c["Rd"]) / out["pi"]
        # the final diagnosis: (w, eta_dot) of the bc output -> its w, u, v
        ws, nb = core.workspace(_lib.WS_SPLIT_VJP)
        wb = core.new("w")
        w_bar, e_bar = cz("w"), cz("eta_dot")  # held: a temporary's memory could be handed to the next one
        check(core.lib.sisl_split_diagnose_vjp(core.handle, w_bar.data_ptr(), e_bar.data_ptr(), g["u"].data_ptr(),
                                               g["v"].data_ptr(), wb.data_ptr(), ws.data_ptr(), nb, core.stream),
              "sisl_split_diagnose_vjp")
        g["w"] = wb
        g["eta_dot"] = torch.zeros_like(wb)
        g["rho"] = torch.zeros_like(rb)
        # bc_fn^T
        if leaves is not None:
            outs, gs = [], []
            for k in pre:
                if torch.is_tensor(post.get(k)) and post[k].requires_grad:
                    outs.append(post[k])
                    gs.append(g[k].to(post[k].dtype).reshape(post[k].shape))
            grads = torch.autograd.grad(outs, [leaves[k] for k in pre], gs, allow_unused=True) if outs else []
            g = {k: (f(gk, locs[k]) if gk is not None else torch.zeros_like(f(pre[k], locs[k])))
                 for k, gk in zip(pre, grads)} if outs else {k: torch.zeros_like(f(pre[k], locs[k])) for k in pre}
        # the three stages
        ob = {"u": g["u"], "v": g["v"], "w": g["w"], "eta_dot": g["eta_dot"], "pi_p": g["pi"], "th_p": g["th_v"]}
        ib = self.step_vjp_device(core, din, ob)
        # the input diagnosis: (w, eta_dot) of the diagnosed input -> the input's w, u, v
        gu, gv = ib["u"].clone(), ib["v"].clone()
        gw = core.new("w")
        check(core.lib.sisl_split_diagnose_vjp(core.handle, ib["w"].data_ptr(), ib["eta_dot"].data_ptr(),
                                               gu.data_ptr(), gv.data_ptr(), gw.data_ptr(), ws.data_ptr(), nb,
                                               core.stream), "sisl_split_diagnose_vjp")
        grads = {"u": gu, "v": gv, "w": gw, "eta_dot": torch.zeros_like(gw), "pi": ib["pi_p"], "th_v": ib["th_p"],
                 "rho": g["rho"] if leaves is None else g.get("rho", torch.zeros_like(rb))}
        return out, grads

    def device_state(self, core, state):
        """The diagnosed device state ``step_device`` and ``step_vjp_device``
        take (u, v, w, eta_dot, pi_p, th_p, rho in the core's layout) from a
        reference-style state dict (u, v, w, pi, th_v, rho)."""
        ph = self.physics
        f = core.field
        u, v = f(state["u"], "u"), f(state["v"], "v")
        eta, w = self._diagnose(core, u, v, f(state["w"], "w"))
        pi_p = fortran(torch.as_tensor(state["pi"]).to(core.device, F64) - ph.pi_bg, dtype=core.dtype)
        th_p = fortran(torch.as_tensor(state["th_v"]).to(core.device, F64) - ph.theta_bg, dtype=core.dtype)
        return {"u": u, "v": v, "w": w, "eta_dot": eta, "pi_p": pi_p, "th_p": th_p, "rho": f(state["rho"], "m")}

    def step(self, state, t, forcing, bc_fn, ml_params=None):
        """SplitExplicitStepper3D.step (steppers.py:1117-1270).  As in the
        reference, the input dict receives the diagnosed eta_dot and w."""
        from .steppers import _dtype_of
        ph, op = self.physics, self.physics.op
        if "rho" not in state:
            raise ValueError("the split-explicit step needs the density 'rho' in the state")
        dtype = _dtype_of({k: state[k] for k in ("u", "v", "w")})
        core = self.core(dtype)
        f = core.field
        u, v = f(state["u"], "u"), f(state["v"], "v")
        eta, w = self._diagnose(core, u, v, f(state["w"], "w"))
        state["eta_dot"], state["w"] = eta, w
        pi_p = fortran(torch.as_tensor(state["pi"]).to(core.device, F64) - ph.pi_bg, dtype=dtype)
        th_p = fortran(torch.as_tensor(state["th_v"]).to(core.device, F64) - ph.theta_bg, dtype=dtype)
        rho = f(state["rho"], "m")
        suite = ph.physics_suite
        bg = ph.precompute_bg(ph.bg_state_ref()) if suite is not None else None  # read by the suite only
        phys = None
        if suite is not None:  # steppers.py:1152-1173
            sp = {"u": u, "v": v, "w": w, "th_v": f(state["th_v"], "m"), "pi": pi_p, "eta_dot": eta,
                  "th_v_prime_u": op.avg(th_p, 0, "m", "u"), "th_v_prime_v": op.avg(th_p, 1, "m", "v"),
                  "th_v_prime_w": op.avg(th_p, 2, "m", "w")}
            for k in state:
                if k not in sp:
                    sp[k] = state[k]
            pt = suite.get_explicit_tendencies(sp, bg, interior_mask=ph.interior_mask, ml_params=ml_params)
            phys = [f(pt[k], loc) if k in pt else None for k, loc in LOCS4]
        st = {"u": u, "v": v, "w": w, "eta_dot": eta, "pi_p": pi_p, "th_p": th_p, "rho": rho}
        res = self.step_device(core, st, phys)
        sn = dict(state)
        sn.pop("_sisl_state", None)
        sn.update({"u": res["u"], "v": res["v"], "w": res["w"], "eta_dot": res["eta_dot"],
                   "pi": fortran(res["pi_p"].double() + ph.pi_bg, dtype=dtype),
                   "th_v": fortran(res["th_p"].double() + ph.theta_bg, dtype=dtype), "rho": rho})
        eps = ph.c.get("eps", 1e-15)
        if suite is not None:  # steppers.py:1233-1247
            state_t = {"u": u, "v": v, "eta_dot": eta}
            for key in suite.tracer_keys:
                if key in state:
                    rq = self.ffsl_advector.advect_3d_split(rho * f(state[key], "m"), state_t, bg)
                    sn[key] = rq / (sn["rho"] + eps)
            sn = suite.apply_state_updates(sn)
        if isinstance(bc_fn, LateralRelaxation):
            sn = bc_fn.apply_state(sn, ph)
        elif bc_fn is not None:
            sn = bc_fn(sn, forcing)
        sn["eta_dot"], sn["w"] = self._diagnose(core, f(sn["u"], "u"), f(sn["v"], "v"), f(sn["w"], "w"))
        tmass = {}
        if suite is not None:
            tmass = {k: sn["rho"] * sn[k] for k in suite.tracer_keys if k in sn}
        sn["rho"] = self._eos(core, sn["th_v"], sn["pi"])
        for k, rq in tmass.items():
            sn[k] = rq / (sn["rho"] + eps)
        return sn
