"""``Simulation`` (shared/driver.py:7-132) on the CPU with a toy step: the
chunking, the step indices and times it passes, the per-chunk metric
report, and the chunk-checkpointed gradient of ``run_differentiable``."""

import math

import torch

from suetes_b200 import Simulation


def test_run_chunks_steps_and_metrics():
    seen, logs = [], []

    def step(state, idx):
        seen.append(idx)
        return {"x": state["x"] + 1.0, "w": state["w"] * 0.5}, state["w"]

    sim = Simulation(step, dt=2.0)
    out = sim.run({"x": torch.zeros(3), "w": torch.full((3,), -8.0)}, 10.0, 10.0 + 2.0 * 7, chunk_steps=3,
                  log=logs.append)
    assert seen == list(range(5, 12))  # int(t_start / dt) onwards, 7 steps
    assert torch.equal(out["x"], torch.full((3,), 7.0))
    progress = [l for l in logs if "Progress" in l]
    assert len(progress) == 2 and "Max W: 8.0000" in progress[0] and "Max W: 1.0000" in progress[1]
    assert any("Finishing remaining 1 steps" in l for l in logs)


def test_run_differentiable_gradient_through_checkpointed_chunks():
    times = []

    def step(state, t, forcing=None, bc_fn=None):
        times.append(t)
        a = 1.0 - 0.01 * t
        out = {"u": a * state["u"] + 0.1 * torch.sin(state["u"]), "is_first_step": 0.0}
        return bc_fn(out, forcing) if bc_fn else out

    u0 = torch.linspace(0.1, 1.0, 5, dtype=torch.float64, requires_grad=True)
    sim = Simulation(step, dt=0.5)
    out = sim.run_differentiable({"u": u0, "is_first_step": 1.0}, 1.0, 1.0 + 0.5 * 7, chunk_steps=3,
                                 bc_fn=lambda s, f: s)
    assert out["is_first_step"] == 0.0
    (g,) = torch.autograd.grad(out["u"].sum(), u0)
    # the same map without chunks or checkpoints
    u = u0.detach().clone().requires_grad_(True)
    v = u
    for n in range(7):
        t = (2 + n) * 0.5
        v = (1.0 - 0.01 * t) * v + 0.1 * torch.sin(v)
    (g_ref,) = torch.autograd.grad(v.sum(), u)
    assert torch.allclose(g, g_ref, rtol=1e-13, atol=0)
    assert math.isclose(times[0], 1.0) and len(set(times)) == 7
    # 7 forward steps, then the two 3-step chunks run again in the backward
    # pass (checkpointed); the 1-step remainder is not checkpointed
    assert len(times) == 7 + 6
    assert sorted(times[7:]) == sorted(times[:6])
