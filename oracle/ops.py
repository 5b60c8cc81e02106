"""Oracle restatement of the C-grid operators and the SL interpolators.

Follows ``suetes/regional3d/operators.py:12-209`` and the trilinear
``jax.scipy.ndimage.map_coordinates(order=1, mode='nearest')`` used at
``suetes/regional3d/steppers.py:367``.  Test infrastructure only.
"""

import torch

from . import DTYPE


class CGridOperator3D:
    """Staggered 2-point differences/averages (operators.py:12-132)."""

    def __init__(self, grid, periodic_axes=()):
        invalid = set(periodic_axes) - {0, 1}
        if invalid:  # operators.py:23-27
            raise ValueError("Only horizontal axes 0 (x) and 1 (y) may be periodic")
        self.grid = grid
        self.periodic_axes = frozenset(periodic_axes)
        self.use_stop_grad = True
        self.m_factors = {loc: m[..., None] for loc, m in grid.m_factors.items()}

    def _apply_padding(self, f, axis, from_loc, to_loc):  # operators.py:37-63
        if from_loc == "m" and to_loc in ("u", "v", "w"):
            n = f.shape[axis]
            left = f.narrow(axis, 0, 1)
            right = f.narrow(axis, n - 1, 1)
            if self.use_stop_grad:
                left, right = left.detach(), right.detach()
            return torch.cat([left, f, right], dim=axis)
        return f

    def diff(self, f, axis, from_loc, to_loc):  # operators.py:65-103
        delta = self.grid.delta[axis]
        d = torch.diff(f, dim=axis) / delta
        if axis in self.periodic_axes and from_loc == "m" and to_loc in ("u", "v"):
            first = f.select(axis, 0)
            last = f.select(axis, f.shape[axis] - 1)
            b = ((first - last) / delta).unsqueeze(axis)
            d = torch.cat([b, d, b], dim=axis)
        else:
            d = self._apply_padding(d, axis, from_loc, to_loc)
        if axis in (0, 1):
            d = d * self.m_factors[to_loc]
        return d

    def avg(self, f, axis, from_loc, to_loc):  # operators.py:105-132
        n = f.shape[axis]
        a = 0.5 * (f.narrow(axis, 0, n - 1) + f.narrow(axis, 1, n - 1))
        if axis in self.periodic_axes and from_loc == "m" and to_loc in ("u", "v"):
            first = f.select(axis, 0)
            last = f.select(axis, n - 1)
            b = (0.5 * (first + last)).unsqueeze(axis)
            return torch.cat([b, a, b], dim=axis)
        return self._apply_padding(a, axis, from_loc, to_loc)


def cubic_weight(p0, p1, p2, p3, t):  # operators.py:134-144
    return ((-0.5 * p0 + 1.5 * p1 - 1.5 * p2 + 0.5 * p3) * t ** 3
            + (p0 - 2.5 * p1 + 2.0 * p2 - 0.5 * p3) * t ** 2
            + (-0.5 * p0 + 0.5 * p2) * t + p1)


def tensor_product_interp_3d(field, coords, use_limiter=False):
    """Catmull-Rom tricubic with clamped stencil (operators.py:146-209)."""
    nx, ny, nz = field.shape
    x = torch.clamp(coords[0], 0, nx - 1)
    y = torch.clamp(coords[1], 0, ny - 1)
    z = torch.clamp(coords[2], 0, nz - 1)
    x0, y0, z0 = (torch.floor(c).to(torch.int64) for c in (x, y, z))
    dx, dy, dz = x - x0, y - y0, z - z0

    def stencil(idx, mx):  # operators.py:176-177
        return (torch.clamp(idx - 1, min=0), idx,
                torch.clamp(idx + 1, max=mx), torch.clamp(idx + 2, max=mx))

    ix, iy, iz = stencil(x0, nx - 1), stencil(y0, ny - 1), stencil(z0, nz - 1)

    def interp_z(xi, yi):
        p = [field[xi, yi, iz[q]] for q in range(4)]
        return cubic_weight(*p, dz)

    def interp_y(xi):
        p = [interp_z(xi, iy[q]) for q in range(4)]
        return cubic_weight(*p, dy)

    vals = [interp_y(ix[q]) for q in range(4)]
    f = cubic_weight(*vals, dx)
    if use_limiter:  # operators.py:192-207
        x1 = torch.clamp(x0 + 1, max=nx - 1)
        y1 = torch.clamp(y0 + 1, max=ny - 1)
        z1 = torch.clamp(z0 + 1, max=nz - 1)
        fmin = fmax = field[x0, y0, z0]
        for i, j, k in [(x1, y0, z0), (x0, y1, z0), (x1, y1, z0), (x0, y0, z1),
                        (x1, y0, z1), (x0, y1, z1), (x1, y1, z1)]:
            nb = field[i, j, k]
            fmin = torch.minimum(fmin, nb)
            fmax = torch.maximum(fmax, nb)
        return torch.minimum(torch.maximum(f, fmin), fmax)
    return f


def map_coordinates_linear(field, coords):
    """``map_coordinates(field, coords, order=1, mode='nearest')``.

    JAX's order-1 path takes ``floor(c)`` and ``floor(c)+1`` with weights
    ``1-(c-floor c)`` and ``c-floor c`` and clips each *index* into
    ``[0, n-1]`` for mode 'nearest'; corner contributions are summed in
    ``itertools.product`` order over the dimensions.  Works for any rank.
    """
    nd = field.dim()
    lowers, ws = [], []
    for d in range(nd):
        c = coords[d]
        lo = torch.floor(c)
        ws.append(c - lo)
        lowers.append(lo.to(torch.int64))
    out = None
    for corner in range(1 << nd):
        idx, w = [], None
        for d in range(nd):
            up = (corner >> (nd - 1 - d)) & 1
            n = field.shape[d]
            i = torch.clamp(lowers[d] + up, 0, n - 1)
            wd = ws[d] if up else (1.0 - ws[d])
            w = wd if w is None else w * wd
            idx.append(i)
        contrib = w * field[tuple(idx)]
        out = contrib if out is None else out + contrib
    return out
