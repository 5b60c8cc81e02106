"""C-grid operators and the tricubic interpolator.

``CGridOperator3D`` mirrors ``suetes/regional3d/operators.py:12-132``: its
``diff``/``avg`` helpers are provided for user scripts (diagnostics, initial
states) and run as plain tensor arithmetic; the step never calls them -- the
CUDA kernels inline the same staggered stencils.  ``tensor_product_interp_3d``
(operators.py:146-209) runs the sm_100a tricubic kernel.
"""

import ctypes

import torch

from . import _lib
from ._lib import check
from .core import DTYPE_CODE, empty_field, fortran, stream_ptr


class CGridOperator3D:
    """Staggered 2-point differences and averages (operators.py:12-132)."""

    def __init__(self, grid, periodic_axes=()):
        if set(periodic_axes) - {0, 1}:
            raise ValueError("Only horizontal axes 0 (x) and 1 (y) may be periodic")
        self.grid = grid
        self.periodic_axes = frozenset(periodic_axes)
        self.use_stop_grad = True
        self.m_factors = {loc: m[..., None] for loc, m in grid.m_factors.items()}

    def _apply_padding(self, f, axis, from_loc, to_loc):
        if from_loc == "m" and to_loc in ("u", "v", "w"):
            n = f.shape[axis]
            return torch.cat([f.narrow(axis, 0, 1), f, f.narrow(axis, n - 1, 1)], dim=axis)
        return f

    def diff(self, f, axis, from_loc, to_loc):
        delta = self.grid.delta[axis]
        d = torch.diff(f, dim=axis) / delta
        if axis in self.periodic_axes and from_loc == "m" and to_loc in ("u", "v"):
            b = ((f.select(axis, 0) - f.select(axis, f.shape[axis] - 1)) / delta).unsqueeze(axis)
            d = torch.cat([b, d, b], dim=axis)
        else:
            d = self._apply_padding(d, axis, from_loc, to_loc)
        if axis in (0, 1):
            d = d * self.m_factors[to_loc].to(d.dtype)
        return d

    def avg(self, f, axis, from_loc, to_loc):
        n = f.shape[axis]
        a = 0.5 * (f.narrow(axis, 0, n - 1) + f.narrow(axis, 1, n - 1))
        if axis in self.periodic_axes and from_loc == "m" and to_loc in ("u", "v"):
            b = (0.5 * (f.select(axis, 0) + f.select(axis, n - 1))).unsqueeze(axis)
            return torch.cat([b, a, b], dim=axis)
        return self._apply_padding(a, axis, from_loc, to_loc)


def _coords3(coords, dtype, device):
    if torch.is_tensor(coords) and coords.dim() == 4:
        cs = [coords[q] for q in range(3)]
    else:
        cs = list(coords)
    return [fortran(c, dtype=dtype, device=device) for c in cs]


def tensor_product_interp_3d(field, coords, use_limiter=False):
    """Catmull-Rom tricubic at continuous indices (operators.py:146-209).

    ``field`` is a 3-D CUDA tensor; ``coords`` a (3, ...) tensor or a
    sequence of three 3-D tensors of the output shape."""
    if not torch.is_tensor(field) or field.device.type != "cuda":
        raise RuntimeError("tensor_product_interp_3d runs on CUDA tensors only")
    f = fortran(field)
    cs = _coords3(coords, f.dtype, f.device)
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
