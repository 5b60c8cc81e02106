"""Host logic of the physics-suite hooks (CPU): the suite's aggregation
(suetes/physics/base.py:28-69) and the relaxation blend on a state dict."""

import torch

from suetes_b200 import LateralRelaxation, PhysicsSuite


class _A:
    def get_tendencies(self, state, bg):
        return {"u": state["u"] * 2.0, "q": state["th_v"] * 0.5}


class _ML:
    is_ml_closure = True

    def get_tendencies(self, state, bg, ml_params=None):
        return {"u": ml_params["c"] + 0.0 * state["u"], "th_v": state["th_v"] - bg["th_v"]}


class _Up:
    def __init__(self, k, f):
        self.k, self.f = k, f

    def apply_update(self, state):
        return {self.k: self.f(state)}


def test_suite_aggregates_masks_and_orders_updates():
    g = torch.Generator().manual_seed(0)
    st = {k: torch.randn(*s, generator=g, dtype=torch.float64) for k, s in
          (("u", (5, 4, 3)), ("v", (4, 5, 3)), ("w", (4, 4, 4)), ("th_v", (4, 4, 3)))}
    bg = {"th_v": torch.full((4, 4, 3), 0.25, dtype=torch.float64)}
    s = PhysicsSuite()
    s.add_tendency_scheme(_A())
    s.add_tendency_scheme(_ML())
    s.register_tracer("q")
    s.register_tracer("q")
    assert s.tracer_keys == ["q"]
    mask = {"u": torch.linspace(0, 1, 5, dtype=torch.float64)[:, None, None]}
    t = s.get_explicit_tendencies(st, bg, interior_mask=mask, ml_params={"c": 3.0})
    assert torch.equal(t["u"], (st["u"] * 2.0 + 3.0) * mask["u"])
    assert torch.equal(t["th_v"], st["th_v"] - bg["th_v"])
    assert torch.equal(t["q"], st["th_v"] * 0.5)
    assert torch.equal(t["v"], torch.zeros_like(st["v"])) and torch.equal(t["w"], torch.zeros_like(st["w"]))
    s.add_update_scheme(_Up("u", lambda x: x["u"] + 1.0))
    s.add_update_scheme(_Up("u", lambda x: x["u"] * 2.0))  # sees its predecessor's result
    out = s.apply_state_updates(st)
    assert torch.equal(out["u"], (st["u"] + 1.0) * 2.0) and out["v"] is st["v"]


def test_relaxation_blend_on_state_dict():
    class Ph:
        theta_bg = torch.full((4, 3, 2), 300.0, dtype=torch.float64)
        pi_bg = torch.full((4, 3, 2), 0.9, dtype=torch.float64)
    mm = torch.rand(4, 3, dtype=torch.float64)
    mu = torch.rand(5, 3, dtype=torch.float64)
    mv = torch.rand(4, 4, dtype=torch.float64)
    r = LateralRelaxation(mm, mu, mv, exterior={"u": 7.0, "v": 0.0, "th_v": 1.5, "pi": 0.0})
    st = {"u": torch.randn(5, 3, 2, dtype=torch.float64), "v": torch.randn(4, 4, 2, dtype=torch.float64),
          "th_v": 300.0 + torch.randn(4, 3, 2, dtype=torch.float64), "pi": torch.full((4, 3, 2), 0.91),
          "w": torch.randn(4, 3, 3, dtype=torch.float64)}
    out = r.apply_state(st, Ph)
    m = mu[..., None]
    assert torch.allclose(out["u"], (1 - m) * st["u"] + m * 7.0, rtol=0, atol=1e-14)
    m = mm[..., None]
    assert torch.allclose(out["th_v"], (1 - m) * st["th_v"] + m * 301.5, rtol=0, atol=1e-12)
    assert torch.allclose(out["pi"].double(), (1 - m) * 0.91 + m * 0.9, rtol=0, atol=1e-7)
    assert out["pi"].dtype == st["pi"].dtype and out["w"] is st["w"]


def test_davies_sponge_inflow_outflow():
    """tests/test_dynamical_core_3d.py:282-333: with a 10 m/s westerly the
    west edge (inflow) relaxes fully to the exterior, the east edge
    (outflow) keeps (1 - outflow_factor) of the model state, the interior
    is untouched; non-blended fields pass through."""
    from suetes_b200 import DaviesSponge

    class G:
        nx, ny, nz = 32, 32, 15

    class Op:
        periodic_axes = ()
    nx, ny, nz = 32, 32, 15
    sp = DaviesSponge(G, Op, sponge_depth=5, dt=30.0, outflow_factor=0.01)
    f64 = torch.float64
    model = {"u": torch.full((nx + 1, ny, nz), 10.0, dtype=f64), "v": torch.zeros(nx, ny + 1, nz, dtype=f64),
             "w": torch.zeros(nx, ny, nz + 1, dtype=f64), "th_v": torch.full((nx, ny, nz), 300.0, dtype=f64),
             "pi": torch.ones(nx, ny, nz, dtype=f64), "q": torch.zeros(nx, ny, nz, dtype=f64)}
    ext = {k: (torch.zeros_like(v) if k in ("u", "v", "w", "q") else v.clone()) for k, v in model.items()}
    out = sp.blend(model, ext)
    assert abs(float(out["u"][nx // 2, ny // 2, nz // 2]) - 10.0) < 1e-12
    assert abs(float(out["u"][0, ny // 2, nz // 2])) < 1e-12
    assert abs(float(out["u"][-1, ny // 2, nz // 2]) - 0.99 * 10.0) < 1e-6
    assert out["w"] is model["w"]
    mask = sp.get_interior_mask()
    assert mask["u"].shape == (nx + 1, ny, 1) and mask["th_v"].shape == (nx, ny, 1)
    assert float(mask["th_v"][nx // 2, ny // 2, 0]) == 1.0 and float(mask["u"][0, ny // 2, 0]) == 0.0


def test_benchmark_sponge_masks_and_blend():
    """boundaries.py:122-190: cos^2 weights on the outer sponge_depth cells,
    combined over x and y, edge-padded to the faces."""
    import math
    from suetes_b200 import BenchmarkSponge
    sp = BenchmarkSponge(12, 10, sponge_depth=3, axes=("x", "y"))
    assert sp.mask_m.shape == (12, 10, 1) and sp.mask_u.shape == (13, 10, 1) and sp.mask_v.shape == (12, 11, 1)
    assert float(sp.mask_m[0, 5, 0]) == 1.0 and float(sp.mask_m[6, 5, 0]) == 0.0
    w1 = math.cos(0.5 * math.pi / 3) ** 2
    assert abs(float(sp.mask_m[1, 5, 0]) - w1) < 1e-6
    assert abs(float(sp.mask_m[1, 1, 0]) - (1 - (1 - w1) ** 2)) < 1e-6
    assert torch.equal(sp.mask_u[-1], sp.mask_u[-2])
    st = {"u": torch.ones(13, 10, 4, dtype=torch.float64), "x_other": torch.ones(3)}
    out = sp.blend(st, {"u": torch.zeros(13, 10, 4, dtype=torch.float64)})
    assert float(out["u"][0, 5, 0]) == 0.0 and float(out["u"][6, 5, 0]) == 1.0 and out["x_other"] is st["x_other"]
    slab = BenchmarkSponge(12, None, sponge_depth=3)
    assert slab.mask_m.shape == (12, 1, 1) and "w" not in slab.blend_vars


def test_cubic_weight_matches_the_oracle():
    from oracle.ops import cubic_weight as ocw
    from suetes_b200.operators import cubic_weight
    g = torch.Generator().manual_seed(3)
    p = [torch.randn(50, generator=g, dtype=torch.float64) for _ in range(4)]
    t = torch.rand(50, generator=g, dtype=torch.float64)
    assert torch.allclose(cubic_weight(*p, t), ocw(*p, t), rtol=1e-13, atol=1e-13)
    assert float(cubic_weight(1.0, 2.0, 3.0, 4.0, 0.0)) == 2.0 and float(cubic_weight(1.0, 2.0, 3.0, 4.0, 1.0)) == 3.0
