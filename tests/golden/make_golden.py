"""Generate the seeded float64 golden fixtures from the CPU oracle.

The reference ships no golden vectors and JAX cannot run here, so these
fixtures are produced by the oracle restatement (pinned by the reference's
known-answer tests, tests/test_oracle_pins.py).  They freeze the oracle's
outputs for small seeded cases; tests/test_golden.py checks that the oracle
still reproduces them (CPU) and that the CUDA path matches them (GPU).

Run from the repository root:  python tests/golden/make_golden.py
"""

import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from _cases import build, mountain, random_fields, shapes5  # noqa: E402

NX, NY, NZ, DT = 10, 8, 6, 20.0


def cases():
    from oracle.steppers import SemiLagrangianAdvector3D, SISLStepper3D, VerticalPreconditioner
    from oracle.ops import tensor_product_interp_3d
    out = {}
    g, op, ph = build("oracle", NX, NY, NZ, 2000.0, 2000.0, 500.0, h=mountain, dt=DT, N_bv=0.01,
                      nu_h_factor=0.05, nu_div_factor=0.1)
    bg = ph.precompute_bg(ph.bg_state_ref())
    x = random_fields(shapes5(NX, NY, NZ), 1234, {"u": 0.1, "v": 0.1, "w": 0.01, "pi": 1e-3, "eta_dot": 1e-3})
    for k, v in x.items():
        out[f"x_{k}"] = v
    L = ph.linear_operator(x, bg, DT, alpha=0.55)
    for k, v in L.items():
        out[f"L_{k}"] = v
    pre = VerticalPreconditioner(ph, DT, alpha=0.55)
    pre.precompute_banded(bg)
    r = random_fields(shapes5(NX, NY, NZ), 4321, {"u": 0.1, "v": 0.1, "w": 0.01, "pi": 1.0, "eta_dot": 0.1})
    for k, v in r.items():
        out[f"r_{k}"] = v
    for k, v in pre(r).items():
        out[f"M_{k}"] = v
    gen = torch.Generator().manual_seed(77)
    f = torch.randn(NX, NY, NZ, generator=gen, dtype=torch.float64)
    co = torch.stack([torch.rand((7, 5, 4), generator=gen, dtype=torch.float64) * (n + 2) - 1 for n in f.shape])
    out["tri_field"], out["tri_coords"] = f, co
    out["tri_out"] = tensor_product_interp_3d(f, co)
    out["tri_out_lim"] = tensor_product_interp_3d(f, co, use_limiter=True)
    s = random_fields({"u": (NX + 1, NY, NZ), "v": (NX, NY + 1, NZ), "eta_dot": (NX, NY, NZ + 1)}, 55,
                      {"u": 20.0, "v": 20.0, "eta_dot": 0.02})
    for k, v in s.items():
        out[f"traj_{k}"] = v
    adv = SemiLagrangianAdvector3D(g, ph, DT)
    for loc in "muvw":
        out[f"dep_{loc}"] = adv.compute_departure_indices(s, loc=loc)
    # one full step from a bubble + wind state
    X, Y, Z = torch.meshgrid(g.x_m, g.y_m, g.z_m, indexing="ij")
    rr = torch.sqrt(X ** 2 + Y ** 2 + (Z - 1500.0) ** 2)
    th = ph.theta_bg + torch.where(rr < 2500.0, 1.5 * torch.cos(0.5 * math.pi * rr / 2500.0) ** 2,
                                   torch.zeros_like(rr))
    C = ph.c
    st = {"u": torch.full((NX + 1, NY, NZ), 4.0, dtype=torch.float64),
          "v": torch.full((NX, NY + 1, NZ), -3.0, dtype=torch.float64),
          "w": torch.zeros(NX, NY, NZ + 1, dtype=torch.float64),
          "eta_dot": torch.zeros(NX, NY, NZ + 1, dtype=torch.float64),
          "pi": ph.pi_bg.clone(), "th_v": th,
          "rho": C["p0"] / (C["Rd"] * th) * ph.pi_bg ** (C["cvd"] / C["Rd"])}
    for k, v in st.items():
        out[f"s0_{k}"] = v
    res = SISLStepper3D(ph, DT, alpha=0.55, solver_tol=1e-12, solver_maxiter=50, solver_restart=25).step(
        st, 0.0, None, lambda a, f_: a)
    for k in ("u", "v", "w", "eta_dot", "pi", "th_v", "rho", "tend_th_v_prev"):
        out[f"s1_{k}"] = res[k]
    return {k: v.detach().numpy() for k, v in out.items()}


if __name__ == "__main__":
    d = cases()
    np.savez_compressed(os.path.join(HERE, "sisl_small_f64.npz"), **d)
    print("wrote", len(d), "arrays")
