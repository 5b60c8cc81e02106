"""Lateral relaxation used as ``bc_fn`` on the device.

The mountain-wave runs of the reference blend u, v, th_v, pi (and rho) toward
an exterior state with an x-dependent cos^2 mask
(``benchmarks/physical/schaer_mountain_3d/run.py:104-126``), the same blend
``(1 - mask) f + mask f_ext`` as ``DaviesSponge.blend`` (boundaries.py:185-293).
``LateralRelaxation`` expresses such a blend for the CUDA step: horizontal
masks per stagger and exterior values in perturbation form.
"""

import math

import torch

from . import _lib
from .core import fortran

FIELD_BITS = {"u": _lib.RELAX_U, "v": _lib.RELAX_V, "w": _lib.RELAX_W, "th_v": _lib.RELAX_TH, "pi": _lib.RELAX_PI}
EXT_INDEX = {"u": 0, "v": 1, "w": 2, "th_v": 3, "pi": 4}


class LateralRelaxation:
    """Blend ``fields`` toward exterior values with horizontal masks.

    ``mask_m`` (nx, ny), ``mask_u`` (nx+1, ny) and ``mask_v`` (nx, ny+1) are
    float tensors in [0, 1]; ``exterior`` maps field names to a constant (for
    th_v and pi: the perturbation from the background, 0 for relaxation to
    the background) or to a 3-D tensor.  Density is re-diagnosed from the
    equation of state after the blend, as in steppers.py:1055-1056.
    """

    def __init__(self, mask_m, mask_u, mask_v, fields=("u", "v", "th_v", "pi"), exterior=None):
        self.mask_m, self.mask_u, self.mask_v = mask_m, mask_u, mask_v
        self.fields = tuple(fields)
        self.exterior = dict(exterior or {})
        self._cache = {}

    def c_struct(self, core):
        key = (core.dtype, str(core.device))
        if key not in self._cache:
            f = lambda t: fortran(torch.as_tensor(t), dtype=core.dtype, device=core.device)
            r = _lib.SislRelaxation()
            r.fields = sum(FIELD_BITS[k] for k in self.fields)
            keep = [f(self.mask_m), f(self.mask_u), f(self.mask_v)]
            r.mask_m, r.mask_u, r.mask_v = (t.data_ptr() for t in keep)
            for k, q in EXT_INDEX.items():
                v = self.exterior.get(k, 0.0)
                if torch.is_tensor(v):
                    t = f(v)
                    keep.append(t)
                    r.ext_field[q] = t.data_ptr()
                else:
                    r.ext[q] = float(v)
            self._cache[key] = (r, keep)
        return self._cache[key][0]

    def __call__(self, state, forcing):
        raise RuntimeError("LateralRelaxation is applied inside the CUDA step")

    def apply_state(self, state, physics):
        """The same blend on a reference state dict (full ``th_v`` and
        ``pi``): thermodynamic fields blend as perturbations from the
        background, in float64, as the fused step blends them.  Used where
        other work (a physics suite's state updates) sits between the step
        and the boundary condition."""
        out = dict(state)
        masks = {"u": self.mask_u, "v": self.mask_v, "w": self.mask_m, "th_v": self.mask_m, "pi": self.mask_m}
        bgs = {"th_v": physics.theta_bg, "pi": physics.pi_bg}
        for k in self.fields:
            f = torch.as_tensor(state[k])
            m = torch.as_tensor(masks[k]).to(device=f.device, dtype=torch.float64)[..., None]
            ext = self.exterior.get(k, 0.0)
            ext = ext.to(device=f.device, dtype=torch.float64) if torch.is_tensor(ext) else float(ext)
            bg = bgs[k].to(device=f.device) if k in bgs else 0.0
            val = f.double() - bg
            out[k] = ((1.0 - m) * val + m * ext + bg).to(f.dtype)
        return out


def x_relaxation(grid, width_m, exterior_u, fields=("u", "v", "th_v", "pi")):
    """The cos^2 x-relaxation zone of schaer_mountain_3d/run.py:104-126:
    mask(i) = cos^2(pi d / (2 n)) for boundary distance d < n = round(width/dx),
    edge-padded to the u faces; exterior u = exterior_u, v = 0 and the
    background thermodynamic state."""
    nx, ny = grid.nx, grid.ny
    n = round(width_m / grid.dx)
    i = torch.arange(nx, dtype=torch.float64, device=grid.device)
    d = torch.minimum(i, nx - 1 - i)
    mask = torch.where(d < n, torch.cos(0.5 * math.pi * d / n) ** 2, torch.zeros_like(d))
    mask_u = torch.cat([mask, mask[-1:]])
    mm = mask[:, None].expand(nx, ny)
    mu = mask_u[:, None].expand(nx + 1, ny)
    mv = mask[:, None].expand(nx, ny + 1)
    return LateralRelaxation(mm, mu, mv, fields=fields,
                             exterior={"u": float(exterior_u), "v": 0.0, "th_v": 0.0, "pi": 0.0})
