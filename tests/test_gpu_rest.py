"""Resting atmospheres stay at rest through the CUDA path (the reference's
tests/test_dynamical_core_3d.py:485-539: 50 steps, max |w| < 1e-7), flat and
over an Agnesi mountain, float64 and float32, for the SISL core (graph
integration) and the split-explicit core."""

import pytest
import torch

from _cases import build

pytestmark = pytest.mark.gpu


def _rest(ph, g, dtype):
    z = lambda t: torch.zeros_like(t, dtype=dtype)
    return {"u": z(g.Z_u), "v": z(g.Z_v), "w": z(g.Z_w), "eta_dot": z(g.Z_w), "pi": ph.pi_bg.clone(),
            "th_v": ph.theta_bg.clone(), "rho": ph.bg_state_ref()["rho"].to(dtype)}


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("mountain", [False, True])
def test_sisl_rest_state(dtype, mountain):
    from suetes_b200 import SISLStepper3D
    h = (lambda x, y: 1500.0 / (1.0 + (x ** 2 + y ** 2) / (30000.0 ** 2))) if mountain else None
    g, op, ph = build("cuda", 24, 20, 16, 6000.0, 6000.0, 500.0, lon=5.0, h=h, device="cuda", dt=60.0, N_bv=0.01)
    st = SISLStepper3D(ph, 60.0, solver_tol=1e-8, solver_maxiter=20, solver_restart=20)
    s = st.integrate(_rest(ph, g, dtype), 0.0, 50, None, lambda a, f: a)
    assert float(s["w"].abs().max()) < 1e-7
    assert bool(torch.isfinite(s["pi"]).all())


@pytest.mark.parametrize("mountain", [False, True])
def test_split_rest_state(mountain):
    from suetes_b200 import SplitExplicitStepper3D
    h = (lambda x, y: 1500.0 / (1.0 + (x ** 2 + y ** 2) / (30000.0 ** 2))) if mountain else None
    g, op, ph = build("cuda", 24, 20, 16, 6000.0, 6000.0, 500.0, lon=5.0, h=h, device="cuda", dt=10.0, N_bv=0.01)
    st = SplitExplicitStepper3D(ph, 10.0, ns=6)
    s = _rest(ph, g, torch.float64)
    for n in range(10):
        s = st.step(s, n * 10.0, None, lambda a, f: a)
    assert float(s["w"].abs().max()) < 1e-7
