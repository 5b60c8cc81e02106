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


def _avg_face_to_mass(f, axis):
    n = f.shape[axis]
    return 0.5 * (f.narrow(axis, 0, n - 1) + f.narrow(axis, 1, n - 1))


def _avg_mass_to_face(f, axis, periodic):
    n = f.shape[axis]
    if periodic:
        b = (0.5 * (f.select(axis, 0) + f.select(axis, n - 1))).unsqueeze(axis)
        return torch.cat([b, _avg_face_to_mass(f, axis), b], dim=axis)
    a = _avg_face_to_mass(f, axis)
    return torch.cat([a.narrow(axis, 0, 1), a, a.narrow(axis, n - 2, 1)], dim=axis)


class DaviesSponge:
    """Davies lateral relaxation with directional outflow scaling
    (boundaries.py:13-120): cos^2 weights over ``sponge_depth`` cells from
    each lateral edge, reduced to ``outflow_factor`` where the flow leaves
    the domain, the strongest edge weight blending u, v, th_v, q and pi
    toward the external state.  Torch on the state's device, for use as (or
    inside) a ``bc_fn``; ``get_interior_mask`` is the physics suites'
    ``interior_mask``."""

    BLEND_VARS = ("u", "v", "th_v", "q", "pi")

    def __init__(self, grid, operators, sponge_depth=30, dt=30.0, tau_bndy_factor=10.0, outflow_factor=0.01):
        self.grid, self.op = grid, operators
        self.depth = sponge_depth
        self.outflow_factor = outflow_factor
        self.max_c = dt / (tau_bndy_factor * dt)  # kept for parity with the reference; the blend does not use it
        self.masks = {loc: self._masks(grid.nx, grid.ny, sponge_depth, loc) for loc in ("u", "v", "m")}

    @staticmethod
    def _masks(nx, ny, depth, loc):
        ix = torch.arange(nx + 1 if loc == "u" else nx, dtype=torch.float32)
        iy = torch.arange(ny + 1 if loc == "v" else ny, dtype=torch.float32)
        ox = 0.0 if loc == "u" else 0.5
        oy = 0.0 if loc == "v" else 0.5
        w = lambda d: torch.cos(0.5 * math.pi * torch.clamp(d / depth, 0.0, 1.0)) ** 2
        return {"west": w(ix + ox)[:, None, None], "east": w(nx - (ix + ox))[:, None, None],
                "south": w(iy + oy)[None, :, None], "north": w(ny - (iy + oy))[None, :, None]}

    def get_interior_mask(self):
        out = {}
        for loc in ("u", "v", "m"):
            m = self.masks[loc]
            interior = 1.0 - torch.maximum(torch.maximum(m["west"], m["east"]), torch.maximum(m["south"], m["north"]))
            if loc == "m":
                out["th_v"] = interior
                out["w"] = interior
            else:
                out[loc] = interior
        return out

    def blend(self, intermediate_state, external_state):
        px = 0 in self.op.periodic_axes
        py = 1 in self.op.periodic_axes
        u, v = intermediate_state["u"], intermediate_state["v"]
        out = {}
        for k, f in intermediate_state.items():
            if k not in self.BLEND_VARS or k not in external_state:
                out[k] = f
                continue
            masks = self.masks.get(k, self.masks["m"])
            if k == "u":
                ue, ve = u, _avg_mass_to_face(_avg_face_to_mass(v, 1), 0, px)
            elif k == "v":
                ue, ve = _avg_mass_to_face(_avg_face_to_mass(u, 0), 1, py), v
            else:
                ue, ve = _avg_face_to_mass(u, 0), _avg_face_to_mass(v, 1)
            ud, vd = ue.detach(), ve.detach()  # the directions carry no gradient
            m = {n: t.to(device=f.device, dtype=f.dtype) for n, t in masks.items()}
            one = torch.ones((), dtype=f.dtype, device=f.device)
            of = torch.full((), self.outflow_factor, dtype=f.dtype, device=f.device)
            c = torch.maximum(torch.maximum(m["west"] * torch.where(ud > 0, one, of),
                                            m["east"] * torch.where(ud < 0, one, of)),
                              torch.maximum(m["south"] * torch.where(vd > 0, one, of),
                                            m["north"] * torch.where(vd < 0, one, of)))
            out[k] = (1.0 - c) * f + c * external_state[k]
        return out


class BenchmarkSponge:
    """Symmetric cos^2 relaxation along x and/or y for the benchmark cases
    (boundaries.py:122-190): weight cos^2(pi d / (2 depth)) at boundary
    distance d < depth, combined over the axes as 1 - (1 - w_x)(1 - w_y),
    edge-padded to the u and v faces; ``blend(state, ext)`` relaxes
    ``blend_vars`` toward ``ext``."""

    def __init__(self, nx, ny=None, sponge_depth=10, axes=("x",), blend_vars=None):
        self.nx, self.ny, self.sponge_depth, self.axes = nx, ny, sponge_depth, axes
        if blend_vars is None:
            blend_vars = (["u", "v", "th_v", "pi", "rho", "q_tr"] if ny is None
                          else ["u", "v", "w", "th_v", "pi", "rho", "q_tr"])
        self.blend_vars = list(blend_vars)

        def weight(n, on):
            if not on:
                return torch.zeros(n, dtype=torch.float32)
            i = torch.arange(n, dtype=torch.float32)
            d = torch.minimum(i, n - 1 - i)
            return torch.where(d < sponge_depth, torch.cos(0.5 * math.pi * d / sponge_depth) ** 2,
                               torch.zeros_like(d))
        wx = weight(nx, "x" in axes)
        wy = weight(ny if ny is not None else 1, "y" in axes and ny is not None)
        if ny is not None:
            self.mask_m = (1.0 - (1.0 - wx[:, None]) * (1.0 - wy[None, :]))[:, :, None]
            self.mask_u = torch.cat([self.mask_m, self.mask_m[-1:]], dim=0)
            self.mask_v = torch.cat([self.mask_m, self.mask_m[:, -1:]], dim=1)
        else:
            self.mask_m = wx[:, None, None]
            self.mask_u = torch.cat([self.mask_m, self.mask_m[-1:]], dim=0)
            self.mask_v = self.mask_m
        self.mask_w = self.mask_m

    def blend(self, state_in, ext_state):
        out = {}
        for k, f in state_in.items():
            if k in self.blend_vars and k in ext_state:
                m = {"u": self.mask_u, "v": self.mask_v, "w": self.mask_w}.get(k, self.mask_m)
                m = m.to(device=f.device, dtype=f.dtype)
                out[k] = (1.0 - m) * f + m * ext_state[k]
            else:
                out[k] = f
        return out
