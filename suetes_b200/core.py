"""Device layout helpers and the Python handle of a CUDA SISL core.

Device layout: a 3-D field keeps the reference's shape ``(ex, ey, ez)`` and
index meaning, but is stored x-fastest (strides ``(1, ex, ex*ey)``), i.e. the
Fortran order of the reference array.  ``fortran()`` produces that layout,
``empty_field()`` allocates it; any other strides are converted on entry.
"""

import ctypes

import torch

from . import _lib
from ._lib import LOC, check, ptrs

F32, F64 = torch.float32, torch.float64
DTYPE_CODE = {F32: _lib.SISL_F32, F64: _lib.SISL_F64}


def is_fortran(t):
    if t.dim() == 3:
        ex, ey, _ = t.shape
        return t.stride() == (1, ex, ex * ey) or t.numel() <= 1
    if t.dim() == 2:
        return t.stride() == (1, t.shape[0]) or t.numel() <= 1
    return t.is_contiguous()


def fortran(t, dtype=None, device=None):
    """Return ``t`` (any strides) as an x-fastest tensor of the same shape."""
    t = torch.as_tensor(t)
    if device is not None or dtype is not None:
        t = t.to(device=device if device is not None else t.device, dtype=dtype if dtype is not None else t.dtype)
    if is_fortran(t):
        return t
    if t.dim() == 3:
        return t.permute(2, 1, 0).contiguous().permute(2, 1, 0)
    if t.dim() == 2:
        return t.t().contiguous().t()
    return t.contiguous()


def empty_field(shape, dtype, device):
    ex, ey, ez = shape
    return torch.empty((ez, ey, ex), dtype=dtype, device=device).permute(2, 1, 0)


def zeros_field(shape, dtype, device):
    return empty_field(shape, dtype, device).zero_()


def stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class Core:
    """Owns a ``SislCore`` (precomputed coefficients for one background, dt,
    alpha and precision) plus cached device workspaces."""

    def __init__(self, grid, constants, theta_bg, pi_bg, tau_damp, dtype, dt, alpha, nu_div, nu_h,
                 periodic_axes=(), solver=None, use_limiter=False, departure_iterations=2, rho_bg=None):
        if grid.device.type != "cuda":
            raise RuntimeError("the SISL core runs on CUDA devices only (no CPU fallback)")
        self.lib = _lib.load()
        self.grid, self.dtype, self.device = grid, dtype, grid.device
        self.dt, self.alpha = float(dt), float(alpha)
        g = _lib.SislGrid(grid.nx, grid.ny, grid.nz, int(0 in periodic_axes), int(1 in periodic_axes),
                          DTYPE_CODE[dtype], grid.dx, grid.dy, grid.dz)
        self.sgrid = g
        solver = dict(solver or {})
        p = _lib.SislParams()
        p.dt, p.alpha = float(dt), float(alpha)
        p.g, p.cp, p.Rd, p.cvd, p.p0 = (float(constants[k]) for k in ("g", "cp", "Rd", "cvd", "p0"))
        p.pi_scale = 1000.0
        p.nu_div, p.nu_h = float(nu_div), float(nu_h)
        p.solver_tol = float(solver.get("tol", 1e-4))
        p.solver_atol = float(solver.get("atol", 0.0))
        p.solver_maxiter = int(solver.get("maxiter", 20))
        p.solver_restart = int(solver.get("restart", 20))
        p.solve_method = int(solver.get("method", _lib.SISL_GMRES_BATCHED))
        p.use_limiter = int(bool(use_limiter))
        p.departure_iterations = int(departure_iterations)
        # float32 cores also carry the float64 operator of GMRES iterative refinement
        p.refine = 1 if dtype == F32 else 0
        self.params = p
        f = lambda t: fortran(t, dtype=F64, device=self.device)
        keep = [f(theta_bg), f(pi_bg), f(grid.Z_m), f(grid.dz_m_full), f(grid.dz_w_full), f(grid.z_xi_w),
                f(grid.z_eta_w), f(tau_damp), f(grid.m_factors["m"]), f(grid.m_factors["u"]),
                f(grid.m_factors["v"]), f(grid.f_u), f(grid.f_v), f(grid.dm_dx_m), f(grid.dm_dy_m)]
        # rho_bg None: the library takes the equation of state of theta_bg and pi_bg
        if rho_bg is not None:
            keep.append(f(rho_bg))
        b = _lib.SislBackground(*[t.data_ptr() for t in keep])
        h = ctypes.c_void_p()
        check(self.lib.sisl_core_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(b),
                                        stream_ptr(self.device), ctypes.byref(h)), "sisl_core_create")
        self.handle = h
        self._ws = {}
        self._solver_key = None
        self.theta_bg = fortran(theta_bg, dtype=F64, device=self.device)
        self.pi_bg = fortran(pi_bg, dtype=F64, device=self.device)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.sisl_core_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------------
    def set_solver(self, tol, maxiter, restart, method, atol=0.0):
        key = (float(tol), float(atol), int(maxiter), int(restart), int(method))
        if key != self._solver_key:
            check(self.lib.sisl_core_set_solver(self.handle, key[0], key[1], key[2], key[3], key[4]),
                  "sisl_core_set_solver")
            self.params.solver_restart = key[3]
            self._solver_key = key

    def autotune(self):
        """Choose the Helmholtz kernels' launch shapes by timing (``sisl_autotune``)."""
        ws, n = self.workspace(_lib.WS_GMRES)
        t = _lib.SislTuning()
        check(self.lib.sisl_autotune(self.handle, ws.data_ptr(), n, self.stream, ctypes.byref(t)), "sisl_autotune")
        return t.as_dict()

    def set_tuning(self, matvec_block=0, precond_tile=0, matvec_t_block=0, precond_t_tile=0, **_):
        t = _lib.SislTuning(matvec_block, precond_tile, matvec_t_block, precond_t_tile)
        check(self.lib.sisl_core_set_tuning(self.handle, ctypes.byref(t)), "sisl_core_set_tuning")

    def tuning(self):
        t = _lib.SislTuning()
        check(self.lib.sisl_autotune_query(self.handle, ctypes.byref(t)), "sisl_autotune_query")
        return t.as_dict()

    def set_refinement(self, on):
        """float64 iterative refinement of a float32 core's GMRES (``sisl_core_set_refinement``)."""
        if self.dtype != F32:
            return
        on = int(bool(on))
        if on != getattr(self, "_refine", None):
            check(self.lib.sisl_core_set_refinement(self.handle, on), "sisl_core_set_refinement")
            self._refine = on

    def set_adjoint(self, tol=None, normalize_rhs=True, method=None):
        """Transposed-solve settings (``sisl_core_set_adjoint``); None keeps the forward's."""
        key = (0.0 if tol is None else float(tol), int(bool(normalize_rhs)), -1 if method is None else int(method))
        if key != getattr(self, "_adjoint_key", None):
            check(self.lib.sisl_core_set_adjoint(self.handle, key[0], key[1], key[2]), "sisl_core_set_adjoint")
            self._adjoint_key = key

    def workspace(self, kind):
        n = int(self.lib.sisl_workspace_bytes(self.handle, kind))
        buf = self._ws.get(kind)
        if buf is None or buf.numel() < n:
            buf = torch.empty(max(n, 256), dtype=torch.uint8, device=self.device)
            self._ws[kind] = buf
        return buf, n

    def shape(self, loc):
        return self.grid.shape_of(loc)

    def field(self, t, loc):
        """A device x-fastest tensor of this core's precision for stagger loc."""
        t = fortran(t, dtype=self.dtype, device=self.device)
        if tuple(t.shape) != self.shape(loc):
            raise ValueError(f"field for stagger {loc} must have shape {self.shape(loc)}, got {tuple(t.shape)}")
        return t

    def new(self, loc):
        return empty_field(self.shape(loc), self.dtype, self.device)

    @property
    def stream(self):
        return stream_ptr(self.device)

    def timing_select(self, kernel_class):
        check(self.lib.sisl_timing_select(self.handle, int(kernel_class)), "sisl_timing_select")

    def timing_read(self):
        """(total milliseconds, launches, algorithmic bytes) of the timed class."""
        ms = ctypes.c_double(0.0)
        n = ctypes.c_int64(0)
        b = ctypes.c_double(0.0)
        check(self.lib.sisl_timing_read(self.handle, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(b)),
              "sisl_timing_read")
        return ms.value, n.value, b.value


LOCS5 = ("u", "v", "w", "m", "w")
KEYS5 = ("u", "v", "w", "pi", "eta_dot")


def vec5(core, d, keys=KEYS5):
    return [core.field(d[k], loc) for k, loc in zip(keys, LOCS5)]


def kernel_launches():
    return int(_lib.load().sisl_kernel_launches())
