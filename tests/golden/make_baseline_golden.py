"""Trajectory fixtures of two benchmark configurations from the CPU oracle.

The reference ships no golden vectors and JAX cannot run here; these
fixtures freeze the float64 oracle (pinned by the reference's own
known-answer tests) on the benchmark grids so the CUDA path can be compared
with it over many steps without rerunning the oracle for minutes:

* ``c1``: the 3-D dry warm bubble, 64x64x48, dx = dy = dz = 50 m, dt = 1 s,
  GMRES tol 1e-10 with restart and maxiter 100 (oracle/cases.py
  ``rising_bubble``), states after 2 and 10 steps;
* ``c2w``: a 64x64x80 window of the 256x256x80 mountain wave (same spacing,
  SLEVE coordinate, ridge, physics and x relaxation; oracle/cases.py
  ``mountain_wave``) at GMRES tol 1e-10, restart 30, maxiter 60, states
  after 5 and 20 steps.

Each state is stored as three slices per field (the x-z plane through the
middle row, the y-z plane through the middle column and the horizontal
plane at mid height; pi and th_v as perturbations pi - pi_bg, th_v -
theta_bg) plus every field's full L2 norm.  Run from the repository root:
python tests/golden/make_baseline_golden.py (about ten minutes on 8 cores).
"""

import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELDS = ("u", "v", "w", "eta_dot", "pi_p", "th_p")
OUT = os.path.join(HERE, "sisl_baseline_trajectories_f64.npz")


def slices(f):
    """x-z, y-z and x-y planes through the middle of a 3-D field, flattened."""
    ex, ey, ez = f.shape
    return np.concatenate([f[:, ey // 2, :].ravel(), f[ex // 2, :, :].ravel(), f[:, :, ez // 2].ravel()])


def perturbation_fields(state, ph):
    to = lambda t: t.detach().double().cpu().numpy()
    return {"u": to(state["u"]), "v": to(state["v"]), "w": to(state["w"]), "eta_dot": to(state["eta_dot"]),
            "pi_p": to(state["pi"]) - to(ph.pi_bg), "th_p": to(state["th_v"]) - to(ph.theta_bg)}


def record(out, tag, n, fields):
    for k in FIELDS:
        out[f"{tag}_{n}_{k}_slices"] = slices(fields[k])
        out[f"{tag}_{n}_{k}_norm"] = np.array(np.linalg.norm(fields[k]))


def run(tag, stepper, state, bc, marks, dt):
    out = {}
    for n in range(1, max(marks) + 1):
        t0 = time.time()
        state = stepper.step(state, (n - 1) * dt, None, bc)
        print(f"{tag} step {n}: {time.time() - t0:.1f} s", flush=True)
        if n in marks:
            record(out, tag, n, perturbation_fields(state, stepper.physics))
    return out


def main():
    torch.set_num_threads(os.cpu_count() or 1)
    from oracle.cases import mountain_wave, rising_bubble
    out = {}
    st, s0, bc = rising_bubble(64, 64, 48, solver_tol=1e-10, solver_maxiter=100, solver_restart=100)
    out.update(run("c1", st, s0, bc, (2, 10), 1.0))
    st, s0, bc = mountain_wave(64, 64, 80, solver_tol=1e-10, solver_maxiter=60, solver_restart=30)
    out.update(run("c2w", st, s0, bc, (5, 20), 8.0))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
