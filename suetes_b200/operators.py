"""C-grid operators and the tricubic interpolator.

``CGridOperator3D`` mirrors ``suetes/regional3d/operators.py:12-132``: every
``diff``/``avg`` runs the sm_100a staggered-stencil kernel and is
differentiable, its backward being the transposed stencil, with the edge
padding's ``stop_gradient`` honoured when ``use_stop_grad`` is set
(operators.py:45-61).  ``tensor_product_interp_3d`` (operators.py:146-209)
runs the tricubic kernel; its field cotangent is the scatter of the 64
Catmull-Rom weights (the step stop-gradients the departure points,
steppers.py:764-767).  CUDA tensors only: there is no CPU path.
"""

import ctypes

import torch

from . import _lib
from ._lib import check
from .core import DTYPE_CODE, empty_field, fortran, stream_ptr


def _require_cuda(t, what):
    if not torch.is_tensor(t) or t.device.type != "cuda":
        raise RuntimeError(f"{what} runs on CUDA tensors only (no CPU path)")


def _stagger_call(f, out, op, axis, to_face, periodic, stop_grad, transpose, inv_delta, mult, in_shape):
    sh = (ctypes.c_int32 * 3)(*in_shape)
    check(_lib.load().sisl_stagger(DTYPE_CODE[f.dtype], op, sh, axis, int(to_face), int(periodic), int(stop_grad),
                                   int(transpose), float(inv_delta), mult.data_ptr() if mult is not None else None,
                                   f.data_ptr(), out.data_ptr(), stream_ptr(f.device)), "sisl_stagger")


class _Stagger(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, op, axis, to_face, periodic, stop_grad, inv_delta, mult):
        f = fortran(f)
        shape = list(f.shape)
        oshape = list(shape)
        oshape[axis] += 1 if to_face else -1
        out = empty_field(tuple(oshape), f.dtype, f.device)
        _stagger_call(f, out, op, axis, to_face, periodic, stop_grad, 0, inv_delta, mult, shape)
        ctx.args = (op, axis, to_face, periodic, stop_grad, inv_delta, mult, shape)
        return out

    @staticmethod
    def backward(ctx, g):
        op, axis, to_face, periodic, stop_grad, inv_delta, mult, shape = ctx.args
        g = fortran(g)
        gin = empty_field(tuple(shape), g.dtype, g.device)
        _stagger_call(g, gin, op, axis, to_face, periodic, stop_grad, 1, inv_delta, mult, shape)
        return gin, None, None, None, None, None, None, None


class CGridOperator3D:
    """Staggered 2-point differences and averages (operators.py:12-132)."""

    def __init__(self, grid, periodic_axes=()):
        if set(periodic_axes) - {0, 1}:
            raise ValueError("Only horizontal axes 0 (x) and 1 (y) may be periodic")
        self.grid = grid
        self.periodic_axes = frozenset(periodic_axes)
        self.use_stop_grad = True
        self.m_factors = {loc: m[..., None] for loc, m in grid.m_factors.items()}
        self._mult = {}

    def _map_factor(self, loc, dtype):
        key = (loc, dtype)
        m = self._mult.get(key)
        if m is None:
            m = fortran(self.grid.m_factors[loc], dtype=dtype)
            self._mult[key] = m
        return m

    def _apply(self, f, op, axis, from_loc, to_loc):
        _require_cuda(f, "CGridOperator3D")
        to_face = from_loc == "m" and to_loc in ("u", "v", "w")
        periodic = axis in self.periodic_axes and from_loc == "m" and to_loc in ("u", "v")
        mult = self._map_factor(to_loc, f.dtype) if (op == _lib.SISL_STAGGER_DIFF and axis in (0, 1)) else None
        inv_delta = 1.0 / self.grid.delta[axis]
        return _Stagger.apply(f, op, axis, to_face, periodic, self.use_stop_grad, inv_delta, mult)

    def diff(self, f, axis, from_loc, to_loc):
        """``(f[i+1] - f[i]) / delta`` to the other stagger, edge-padded or
        periodic, times the map factor on horizontal axes (operators.py:65-103)."""
        return self._apply(f, _lib.SISL_STAGGER_DIFF, axis, from_loc, to_loc)

    def avg(self, f, axis, from_loc, to_loc):
        """Two-point average to the other stagger (operators.py:105-132)."""
        return self._apply(f, _lib.SISL_STAGGER_AVG, axis, from_loc, to_loc)


def _coords3(coords, dtype, device):
    if torch.is_tensor(coords) and coords.dim() == 4:
        cs = [coords[q] for q in range(3)]
    else:
        cs = list(coords)
    return [fortran(c, dtype=dtype, device=device) for c in cs]


class _Tricubic(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, use_limiter, scale, *cs):
        out = _tricubic_fwd(field, cs, use_limiter)
        if scale != 1.0:
            out = out * scale
        ctx.save_for_backward(field, *cs)
        ctx.use_limiter, ctx.scale = use_limiter, scale
        return out

    @staticmethod
    def backward(ctx, g):
        field, *cs = ctx.saved_tensors
        grad = tricubic_vjp(field, cs, g, ctx.use_limiter, ctx.scale)
        return (grad, None, None) + (None,) * len(cs)


def tricubic_vjp(field, coords, cot, use_limiter=False, scale=1.0, out=None, deterministic=True):
    """Cotangent of ``field`` for ``scale * tensor_product_interp_3d(field,
    coords)`` given the output cotangent (accumulated into ``out`` when given).

    ``deterministic`` (default) sums the scattered contributions as
    fixed-point integers (``sisl_tricubic_vjp_deterministic``): the result is
    the same bits on every run.  ``False`` scatters with float atomics."""
    f = fortran(field)
    cs = _coords3(coords, f.dtype, f.device)
    g = fortran(cot, dtype=f.dtype)
    if out is None:
        out = empty_field(tuple(f.shape), f.dtype, f.device).zero_()
    src = (ctypes.c_int32 * 3)(*f.shape)
    dst = (ctypes.c_int32 * 3)(*cs[0].shape)
    co = (ctypes.c_void_p * 3)(*[c.data_ptr() for c in cs])
    lib = _lib.load()
    if deterministic:
        nbytes = int(lib.sisl_tricubic_vjp_workspace_bytes(DTYPE_CODE[f.dtype], src))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=f.device)
        check(lib.sisl_tricubic_vjp_deterministic(DTYPE_CODE[f.dtype], src, f.data_ptr(), dst, co, g.data_ptr(),
                                                  out.data_ptr(), int(bool(use_limiter)), float(scale),
                                                  ws.data_ptr(), nbytes, stream_ptr(f.device)),
              "sisl_tricubic_vjp_deterministic")
    else:
        check(lib.sisl_tricubic_vjp(DTYPE_CODE[f.dtype], src, f.data_ptr(), dst, co, g.data_ptr(),
                                    out.data_ptr(), int(bool(use_limiter)), float(scale),
                                    stream_ptr(f.device)), "sisl_tricubic_vjp")
    return out


def cubic_weight(p0, p1, p2, p3, t):
    """The Catmull-Rom cubic through p1, p2 at fraction t (operators.py:134-144),
    as the weights of p0..p3 the tricubic kernel applies (tensors or floats)."""
    w0 = t * (-0.5 + t * (1.0 - 0.5 * t))
    w1 = 1.0 + t * t * (-2.5 + 1.5 * t)
    w2 = t * (0.5 + t * (2.0 - 1.5 * t))
    w3 = t * t * (-0.5 + 0.5 * t)
    return w0 * p0 + w1 * p1 + w2 * p2 + w3 * p3


def tensor_product_interp_3d(field, coords, use_limiter=False):
    """Catmull-Rom tricubic at continuous indices (operators.py:146-209).

    ``field`` is a 3-D CUDA tensor; ``coords`` a (3, ...) tensor or a
    sequence of three 3-D tensors of the output shape.  Differentiable with
    respect to ``field``; coordinates must not require gradients."""
    _require_cuda(field, "tensor_product_interp_3d")
    cs = _coords3(coords, field.dtype, field.device)
    if any(c.requires_grad for c in cs):
        raise NotImplementedError("tensor_product_interp_3d provides no coordinate cotangents "
                                  "(departure points are stop-gradiented, steppers.py:764-767)")
    if torch.is_grad_enabled() and field.requires_grad:
        return _Tricubic.apply(field, bool(use_limiter), 1.0, *cs)
    return _tricubic_fwd(field, cs, use_limiter)


def _tricubic_fwd(field, cs, use_limiter):
    f = fortran(field)
    out = empty_field(tuple(cs[0].shape), f.dtype, f.device)
    src = (ctypes.c_int32 * 3)(*f.shape)
    dst = (ctypes.c_int32 * 3)(*cs[0].shape)
    co = (ctypes.c_void_p * 3)(*[c.data_ptr() for c in cs])
    check(_lib.load().sisl_tricubic(DTYPE_CODE[f.dtype], src, f.data_ptr(), dst, co, out.data_ptr(),
                                    int(bool(use_limiter)), stream_ptr(f.device)), "sisl_tricubic")
    return out


def map_coordinates_linear(field, coords):
    """``map_coordinates(field, coords, order=1, mode='nearest')`` on 3-D fields."""
    f = fortran(field)
    cs = _coords3(coords, f.dtype, f.device)
    out = empty_field(tuple(cs[0].shape), f.dtype, f.device)
    src = (ctypes.c_int32 * 3)(*f.shape)
    dst = (ctypes.c_int32 * 3)(*cs[0].shape)
    co = (ctypes.c_void_p * 3)(*[c.data_ptr() for c in cs])
    check(_lib.load().sisl_trilinear(DTYPE_CODE[f.dtype], src, f.data_ptr(), dst, co, out.data_ptr(),
                                     stream_ptr(f.device)), "sisl_trilinear")
    return out
