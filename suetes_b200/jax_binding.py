"""jax.ffi binding of the SISL library (for hosts with JAX and jaxlib).

The reference steps its state with ``SISLStepper3D.step`` under ``jax.jit``
(suetes/regional3d/steppers.py:720-1073); this module exposes the same step
as XLA FFI custom calls into ``libsisl_xla_ffi.so`` (built by
``make -C suetes_b200/csrc ffi`` from ``suetes_b200/ffi/sisl_xla_ffi.cc``)
with a ``jax.custom_vjp`` whose forward keeps the two implicit solves
(``sisl_step_taped``) and whose backward rule is ``sisl_step_vjp`` -- the
``jax.checkpoint`` + ``custom_linear_solve`` gradient of the reference step.

JAX is not a dependency of this package: importing this module without JAX
raises ImportError.  The coefficient set is a ``suetes_b200.core.Core``
(created with torch on the same device); its handle is passed to the
handlers as an attribute.  Arrays are the device-layout (perturbation-form)
fields of ``DeviceState.FIELDS``, requested x-fastest (layout (0, 1, 2)).
"""

import ctypes
import os

import jax
import jax.numpy as jnp

from . import _lib

STATE_KEYS = ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho", "u_prev", "v_prev", "w_prev", "eta_dot_prev",
              "tend_th_prev")
SOLVE_LOCS = ("u", "v", "w", "m", "w")
_XFAST = (0, 1, 2)
_registered = False


def register(path=None):
    """Load libsisl_xla_ffi.so and register its handlers for the CUDA platform."""
    global _registered
    if _registered:
        return
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsisl_xla_ffi.so")
    lib = ctypes.cdll.LoadLibrary(path)
    for name, sym in (("sisl_step", "SislStep"), ("sisl_step_vjp", "SislStepVjp"),
                      ("sisl_gmres_solve", "SislGmresSolve"), ("sisl_tricubic", "SislTricubic"),
                      ("sisl_tricubic_vjp", "SislTricubicVjp")):
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(lib, sym)), platform="CUDA")
    _registered = True


def _shape(core, loc):
    return tuple(core.shape(loc))


def _state_structs(core, dtype):
    locs = dict(core_locs())
    return [jax.ShapeDtypeStruct(_shape(core, locs[k]), dtype) for k in STATE_KEYS]


def core_locs():
    from .steppers import DeviceState
    return DeviceState.FIELDS


def _ws_struct(core, kind):
    n = int(core.lib.sisl_workspace_bytes(core.handle, kind))
    return jax.ShapeDtypeStruct((n,), jnp.uint8)


def make_step(core, relax_ptr=0):
    """``step(state_tuple, is_first_step) -> state_tuple`` with the custom VJP
    of the reference's differentiable step; ``core`` a suetes_b200 Core."""
    register()
    dtype = jnp.float32 if core.dtype.itemsize == 4 else jnp.float64
    handle = int(core.handle.value)
    outs = _state_structs(core, dtype)
    solves = [jax.ShapeDtypeStruct(_shape(core, l), dtype) for l in SOLVE_LOCS * 2]
    n_in = len(STATE_KEYS)

    def taped(state, first):
        call = jax.ffi.ffi_call("sisl_step", outs + solves + [_ws_struct(core, _lib.WS_STEP)],
                                input_layouts=[_XFAST] * n_in,
                                output_layouts=[_XFAST] * (n_in + 10) + [None])
        res = call(*state, core=handle, relax=relax_ptr, is_first_step=float(first), taped=1)
        return tuple(res[:n_in]), tuple(res[n_in:n_in + 10])

    def vjp_call(state, tape, out_bar, first):
        call = jax.ffi.ffi_call("sisl_step_vjp", outs + [_ws_struct(core, _lib.WS_STEP_VJP)],
                                input_layouts=[_XFAST] * (2 * n_in + 10),
                                output_layouts=[_XFAST] * n_in + [None])
        res = call(*state, *tape, *out_bar, core=handle, relax=relax_ptr, is_first_step=float(first))
        return tuple(res[:n_in])

    def make(first):
        @jax.custom_vjp
        def step(state):
            return taped(state, first)[0]

        def fwd(state):
            out, tape = taped(state, first)
            return out, (state, tape)

        def bwd(res, out_bar):
            state, tape = res
            return (vjp_call(state, tape, out_bar, first),)

        step.defvjp(fwd, bwd)
        return step

    steps = {1.0: make(1.0), 0.0: make(0.0)}
    return lambda state, is_first_step=0.0: steps[float(is_first_step)](tuple(state))
