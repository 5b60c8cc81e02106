"""Committed seeded fixtures (tests/golden/make_golden.py): the oracle must
reproduce them (CPU) and the CUDA float64 path must match them (GPU)."""

import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from _cases import build, mountain  # noqa: E402

G = dict(np.load(os.path.join(HERE, "golden", "sisl_small_f64.npz")))
NX, NY, NZ, DT = 10, 8, 6, 20.0
KW = dict(h=mountain, dt=DT, N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1)


def test_oracle_reproduces_golden():
    import make_golden
    d = make_golden.cases()
    for k, v in G.items():
        assert np.allclose(d[k], v, rtol=1e-12, atol=1e-14 * max(1.0, float(np.abs(v).max()))), k


def _t(k, dev="cuda"):
    return torch.from_numpy(G[k]).to(dev)


@pytest.mark.gpu
def test_cuda_matches_golden():
    import suetes_b200 as sb
    g, op, ph = build("cuda", NX, NY, NZ, 2000.0, 2000.0, 500.0, device="cuda", **KW)
    bg = ph.precompute_bg(ph.bg_state_ref())
    keys = ("u", "v", "w", "pi", "eta_dot")
    L = ph.linear_operator({k: _t(f"x_{k}") for k in keys}, bg, DT, alpha=0.55)
    for k in keys:
        assert np.allclose(L[k].cpu().numpy(), G[f"L_{k}"], rtol=1e-11, atol=1e-13), k
    pre = sb.VerticalPreconditioner(ph, DT, alpha=0.55)
    pre.precompute_banded(bg)
    M = pre({k: _t(f"r_{k}") for k in keys})
    for k in keys:
        ref = G[f"M_{k}"]
        assert np.allclose(M[k].cpu().numpy(), ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max()), k
    co = _t("tri_coords")
    assert np.allclose(sb.tensor_product_interp_3d(_t("tri_field"), co).cpu().numpy(), G["tri_out"], atol=1e-13)
    assert np.allclose(sb.tensor_product_interp_3d(_t("tri_field"), co, use_limiter=True).cpu().numpy(),
                       G["tri_out_lim"], atol=1e-13)
    adv = sb.SemiLagrangianAdvector3D(g, ph, DT)
    s = {k: _t(f"traj_{k}") for k in ("u", "v", "eta_dot")}
    for loc in "muvw":
        assert np.abs(adv.compute_departure_indices(s, loc=loc).cpu().numpy() - G[f"dep_{loc}"]).max() < 1e-12
    st = {k: _t(f"s0_{k}") for k in ("u", "v", "w", "eta_dot", "pi", "th_v", "rho")}
    res = sb.SISLStepper3D(ph, DT, alpha=0.55, solver_tol=1e-12, solver_maxiter=50, solver_restart=25).step(
        st, 0.0, None, lambda a, f_: a)
    for k in ("u", "v", "w", "eta_dot", "rho", "tend_th_v_prev"):
        ref = G[f"s1_{k}"]
        err = np.linalg.norm(res[k].double().cpu().numpy() - ref) / max(np.linalg.norm(ref), 1e-300)
        assert err < 1e-8, (k, err)
    thp = res["_sisl_state"][0].t["th_p"].cpu().numpy()
    ref = G["s1_th_v"] - ph.theta_bg.cpu().numpy()
    assert np.linalg.norm(thp - ref) / np.linalg.norm(ref) < 1e-8
