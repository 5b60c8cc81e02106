"""ctypes binding of the C ABI declared in ``include/sisl_b200.h``.

The shared library ``libsisl_b200.so`` is built in-tree by
``make -C suetes_b200/csrc`` (or ``__graft_entry__.build()``).  There is no
fallback: every numerical entry point of this package goes through this
library, and a missing library raises immediately.
"""

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsisl_b200.so")

SISL_F32, SISL_F64 = 0, 1
LOC = {"m": 0, "u": 1, "v": 2, "w": 3}
SISL_GMRES_BATCHED, SISL_GMRES_INCREMENTAL = 0, 1
WS_STEP, WS_GMRES, WS_DEPARTURE, WS_EXPLICIT, WS_OPERATOR, WS_FFSL = 0, 1, 2, 3, 4, 5
WS_STEP_VJP, WS_EXPLICIT_VJP, WS_FFSL_VJP, WS_SPLIT, WS_SPLIT_VJP = 6, 7, 8, 9, 10
RELAX_U, RELAX_V, RELAX_W, RELAX_TH, RELAX_PI = 1, 2, 4, 8, 16
K_NONE, K_MATVEC, K_PRECOND, K_DOTS, K_UPDATE, K_SL, K_EXPLICIT, K_OTHER = range(8)
SISL_OK, SISL_NOT_CONVERGED = 0, 1
SISL_STAGGER_AVG, SISL_STAGGER_DIFF = 0, 1
SISL_ERR_SCRATCH_LIMIT = -5
FFSL_NOALLOC_MAX_DOUBLES = 1 << 20

c_double_p = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p


class SislGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("periodic_x", ctypes.c_int32), ("periodic_y", ctypes.c_int32), ("dtype", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double)]


class SislParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("alpha", ctypes.c_double), ("g", ctypes.c_double),
                ("cp", ctypes.c_double), ("Rd", ctypes.c_double), ("cvd", ctypes.c_double),
                ("p0", ctypes.c_double), ("pi_scale", ctypes.c_double), ("nu_div", ctypes.c_double),
                ("nu_h", ctypes.c_double), ("solver_tol", ctypes.c_double), ("solver_atol", ctypes.c_double),
                ("solver_maxiter", ctypes.c_int32), ("solver_restart", ctypes.c_int32),
                ("solve_method", ctypes.c_int32), ("use_limiter", ctypes.c_int32),
                ("departure_iterations", ctypes.c_int32), ("refine", ctypes.c_int32)]


class SislBackground(ctypes.Structure):
    _fields_ = [(n, vp) for n in ("theta_bg", "pi_bg", "Z_m", "dz_m_full", "dz_w_full", "z_xi_w", "z_eta_w",
                                  "tau_damp", "m_m", "m_u", "m_v", "f_u", "f_v", "dm_dx_m", "dm_dy_m",
                                  "rho_bg")]


class SislSolveInfo(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_int32), ("arnoldi_steps", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("residual_norm", ctypes.c_double), ("atol", ctypes.c_double),
                ("b_norm", ctypes.c_double)]

    def as_dict(self):
        return {"cycles": self.cycles, "arnoldi_steps": self.arnoldi_steps, "converged": bool(self.converged),
                "residual_norm": self.residual_norm, "atol": self.atol, "b_norm": self.b_norm}


class SislTuning(ctypes.Structure):
    _fields_ = [("matvec_block", ctypes.c_int32), ("precond_tile", ctypes.c_int32),
                ("matvec_t_block", ctypes.c_int32), ("precond_t_tile", ctypes.c_int32),
                ("us", ctypes.c_float * 4)]

    def as_dict(self):
        return {"matvec_block": self.matvec_block, "precond_tile": self.precond_tile,
                "matvec_t_block": self.matvec_t_block, "precond_t_tile": self.precond_t_tile,
                "us": [round(float(x), 2) for x in self.us]}


class SislState(ctypes.Structure):
    _fields_ = [(n, vp) for n in ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho", "u_prev", "v_prev",
                                  "w_prev", "eta_dot_prev", "tend_th_prev")] + [("is_first_step", ctypes.c_double)]


class SislRelaxation(ctypes.Structure):
    _fields_ = [("fields", ctypes.c_int32), ("pad", ctypes.c_int32), ("mask_m", vp), ("mask_u", vp),
                ("mask_v", vp), ("ext", ctypes.c_double * 5), ("ext_field", vp * 5)]


class SislStepInfo(ctypes.Structure):
    _fields_ = [("solve", SislSolveInfo * 2), ("kernel_launches", ctypes.c_int64)]


# name -> (restype, argtypes); the exported symbol set of sisl_b200.h
PROTOTYPES = {
    "sisl_version": (ctypes.c_int, []),
    "sisl_last_error": (ctypes.c_char_p, []),
    "sisl_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sisl_field_elems": (ctypes.c_size_t, [ctypes.POINTER(SislGrid), ctypes.c_int]),
    "sisl_core_create": (ctypes.c_int, [ctypes.POINTER(SislGrid), ctypes.POINTER(SislParams),
                                        ctypes.POINTER(SislBackground), vp, ctypes.POINTER(vp)]),
    "sisl_core_destroy": (ctypes.c_int, [vp]),
    "sisl_core_set_solver": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int]),
    "sisl_core_set_adjoint": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "sisl_core_set_refinement": (ctypes.c_int, [vp, ctypes.c_int]),
    "sisl_workspace_bytes": (ctypes.c_size_t, [vp, ctypes.c_int]),
    "sisl_linear_operator": (ctypes.c_int, [vp, vp * 5, vp * 5, vp, ctypes.c_size_t, vp]),
    "sisl_helmholtz_matvec": (ctypes.c_int, [vp, vp * 5, vp * 5, vp]),
    "sisl_precond_apply": (ctypes.c_int, [vp, vp * 5, vp * 5, vp]),
    "sisl_gmres_solve": (ctypes.c_int, [vp, vp * 5, vp, vp * 5, vp, ctypes.c_size_t, vp,
                                        ctypes.POINTER(SislSolveInfo)]),
    "sisl_helmholtz_matvec_t": (ctypes.c_int, [vp, vp * 5, vp * 5, vp, ctypes.c_size_t, vp]),
    "sisl_precond_apply_t": (ctypes.c_int, [vp, vp * 5, vp * 5, vp]),
    "sisl_gmres_solve_transpose": (ctypes.c_int, [vp, vp * 5, vp, vp * 5, vp, ctypes.c_size_t, vp,
                                                  ctypes.POINTER(SislSolveInfo)]),
    "sisl_departure": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp * 3, vp, ctypes.c_size_t,
                                      vp]),
    "sisl_tricubic": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32 * 3, vp, ctypes.c_int32 * 3, vp * 3, vp,
                                     ctypes.c_int, vp]),
    "sisl_tricubic_vjp": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32 * 3, vp, ctypes.c_int32 * 3, vp * 3, vp, vp,
                                         ctypes.c_int, ctypes.c_double, vp]),
    "sisl_tricubic_vjp_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int32 * 3]),
    "sisl_tricubic_vjp_deterministic": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32 * 3, vp, ctypes.c_int32 * 3,
                                                       vp * 3, vp, vp, ctypes.c_int, ctypes.c_double, vp,
                                                       ctypes.c_size_t, vp]),
    "sisl_stagger": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int32 * 3, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, vp, vp, vp, vp]),
    "sisl_explicit_tendencies": (ctypes.c_int, [vp, vp * 6, vp * 6, vp, vp, ctypes.c_size_t, vp]),
    "sisl_tendencies": (ctypes.c_int, [vp, ctypes.c_int, vp * 6, vp * 6, vp, vp, ctypes.c_size_t, vp]),
    "sisl_metric_curvature": (ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
    "sisl_trilinear": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32 * 3, vp, ctypes.c_int32 * 3, vp * 3, vp, vp]),
    "sisl_ffsl_lines_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    "sisl_ffsl_lines": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp,
                                       ctypes.c_size_t, vp]),
    "sisl_ffsl_lines_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int,
                                               vp, vp]),
    "sisl_ffsl_advect": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "sisl_ffsl_advect_vjp": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "sisl_ffsl_lines_vjp_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    "sisl_ffsl_lines_vjp": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp,
                                           vp, vp, ctypes.c_size_t, vp]),
    "sisl_eos": (ctypes.c_int, [vp, vp, vp, vp, vp]),
    "sisl_step": (ctypes.c_int, [vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState),
                                 ctypes.POINTER(SislRelaxation), vp, ctypes.c_size_t, vp,
                                 ctypes.POINTER(SislStepInfo)]),
    "sisl_step_taped": (ctypes.c_int, [vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState),
                                       ctypes.POINTER(SislRelaxation), vp * 10, vp, ctypes.c_size_t, vp,
                                       ctypes.POINTER(SislStepInfo)]),
    "sisl_step_physics": (ctypes.c_int, [vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState),
                                         ctypes.POINTER(SislRelaxation), vp * 4, vp, vp, ctypes.c_size_t, vp,
                                         ctypes.POINTER(SislStepInfo)]),
    "sisl_split_diagnose": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp]),
    "sisl_split_diagnose_vjp": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "sisl_split_step": (ctypes.c_int, [vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState), ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, vp, vp * 4, vp, ctypes.c_size_t, vp]),
    "sisl_split_step_vjp": (ctypes.c_int, [vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState),
                                           ctypes.POINTER(SislState), ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           vp, ctypes.c_int, vp, ctypes.c_size_t, vp]),
    "sisl_step_vjp": (ctypes.c_int, [vp, ctypes.POINTER(SislState), vp * 10, ctypes.POINTER(SislRelaxation),
                                     ctypes.POINTER(SislState), ctypes.POINTER(SislState), vp, ctypes.c_size_t, vp,
                                     ctypes.POINTER(SislStepInfo)]),
    "sisl_explicit_tendencies_vjp": (ctypes.c_int, [vp, vp * 6, vp * 6, vp, vp * 6, vp, ctypes.c_size_t, vp]),
    "sisl_step_graph_create": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(SislState), ctypes.POINTER(SislState),
                                              vp, vp, vp, vp, ctypes.POINTER(vp)]),
    "sisl_step_graph_create_taped": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(SislState),
                                                    ctypes.POINTER(SislState), vp, vp, vp, vp, vp,
                                                    ctypes.POINTER(vp)]),
    "sisl_step_graph_create_grouped": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(SislState),
                                                      ctypes.POINTER(SislState), vp, vp, vp, vp, vp,
                                                      ctypes.POINTER(vp)]),
    "sisl_step_vjp_graph_create": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(SislState), vp, vp,
                                                  ctypes.POINTER(SislState), ctypes.POINTER(SislState), vp, vp, vp,
                                                  ctypes.POINTER(vp)]),
    "sisl_step_vjp_graph_create_grouped": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(SislState), vp, vp,
                                                          ctypes.POINTER(SislState), ctypes.POINTER(SislState), vp,
                                                          vp, vp, ctypes.POINTER(vp)]),
    "sisl_step_graph_launch": (ctypes.c_int, [vp, vp]),
    "sisl_step_graph_info": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(SislStepInfo), vp]),
    "sisl_step_graph_destroy": (ctypes.c_int, [vp]),
    "sisl_autotune": (ctypes.c_int, [vp, vp, ctypes.c_size_t, vp, ctypes.POINTER(SislTuning)]),
    "sisl_autotune_query": (ctypes.c_int, [vp, ctypes.POINTER(SislTuning)]),
    "sisl_core_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(SislTuning)]),
    "sisl_kernel_launches": (ctypes.c_int64, []),
    "sisl_timing_select": (ctypes.c_int, [vp, ctypes.c_int]),
    "sisl_timing_read": (ctypes.c_int, [vp, c_double_p, ctypes.POINTER(ctypes.c_int64), c_double_p]),
}

_LIB = None


def load():
    """Load ``libsisl_b200.so`` (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -c 'import __graft_entry__ as g; g.build()' or make -C suetes_b200/csrc)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def status_string(rc):
    return load().sisl_status_string(rc).decode()


def check(rc, what):
    """Raise on a negative status; return the status otherwise."""
    if rc < 0:
        detail = ""
        if rc == -2:
            try:
                detail = load().sisl_last_error().decode()
            except Exception:
                detail = ""
        raise RuntimeError(f"{what} failed: {status_string(rc)} (status {rc})" + (f": {detail}" if detail else ""))
    return rc


def ptrs(tensors, n):
    arr = (vp * n)()
    for q, t in enumerate(tensors):
        arr[q] = None if t is None else t.data_ptr()
    return arr
