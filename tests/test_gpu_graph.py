"""CUDA-graph steps (sisl_step_graph_*) against the eager sisl_step.

A graph replays the same kernels in the same order, the GMRES restart loops
as device-decided conditional nodes, so its states must equal the eager
steps bit for bit, with the same solve statistics; members of different
sizes in one graph must each equal their own eager run.
"""

import pytest
import torch

from suetes_b200.workloads import rising_bubble

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho", "u_prev", "tend_th_prev")


def _eager(stepper, ds0, relax, nsteps):
    from suetes_b200 import DeviceState
    core = ds0.core
    cur = DeviceState(core, {k: v.clone() for k, v in ds0.t.items()}, ds0.is_first_step)
    infos = []
    for _ in range(nsteps):
        nxt = DeviceState(core)
        infos.append(stepper.step_device(cur, nxt, relax))
        cur = nxt
    return cur, infos


def _member(n, nz, dtype, amp=2.0, tol=None, maxiter=30, method="batched", ny=None):
    st, s0, bc = rising_bubble(n, ny or n, nz, dx=50.0, amp=amp, dtype=dtype,
                               solver_tol=tol or (1e-10 if dtype == torch.float64 else 1e-7),
                               solver_maxiter=maxiter, solver_restart=30, solve_method=method)
    return st, st.to_device_state(s0), bc


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_graph_steps_equal_eager(dtype):
    from suetes_b200 import PingPong
    st, ds0, bc = _member(24, 16, dtype)
    ref, infos = _eager(st, ds0, bc, 4)
    pp = PingPong([(st, ds0, bc)])
    assert pp.steps_done == 1
    for _ in range(3):
        pp.step()
    out = pp.current()[0]
    for k in FIELDS:
        assert torch.equal(out.t[k], ref.t[k]), k
    gi = pp.info(0)["solves"]
    for q in range(2):
        assert gi[q]["cycles"] == infos[-1]["solves"][q]["cycles"]
        assert gi[q]["arnoldi_steps"] == infos[-1]["solves"][q]["arnoldi_steps"]
        assert gi[q]["converged"]


def test_graph_ensemble_members_equal_their_eager_runs():
    from suetes_b200 import PingPong
    specs = [(16, 12, 1.5), (24, 16, 2.5), (20, 10, 2.0)]
    members = [_member(n, nz, torch.float32, amp=a) for n, nz, a in specs]
    refs = [_eager(st, ds0, bc, 3)[0] for st, ds0, bc in members]
    pp = PingPong(members)
    pp.step()
    pp.step()
    for m, ref in enumerate(refs):
        out = pp.current()[m]
        for k in FIELDS:
            assert torch.equal(out.t[k], ref.t[k]), (m, k)


@pytest.mark.parametrize("dtype,method", [(torch.float32, "batched"), (torch.float32, "incremental"),
                                          (torch.float64, "batched")])
def test_grouped_solves_equal_the_branch_graph(dtype, method):
    """Grouped solves (every Krylov phase one launch over a member/block
    table, one WHILE node per solve) give every member the same bits and
    solve statistics as the graph of per-member branches, with members of
    uneven sizes converging after different cycle counts and one member
    stopped by its maxiter."""
    from suetes_b200 import PingPong
    specs = [(16, 12, 12, 1.5, None, 30), (24, 20, 16, 2.5, None, 30), (20, 20, 10, 2.0, 1e-14, 1)]
    members = [_member(n, nz, dtype, amp=a, tol=tol, maxiter=mi, method=method, ny=ny)
               for n, ny, nz, a, tol, mi in specs]
    branch = PingPong(members)
    grouped = PingPong(members, grouped=True)
    for _ in range(3):
        branch.step()
        grouped.step()
    cycles = []
    for m in range(len(members)):
        a, b = branch.current()[m], grouped.current()[m]
        for k in FIELDS:
            assert torch.equal(a.t[k], b.t[k]), (m, k, (a.t[k] - b.t[k]).abs().max().item())
        ia, ib = branch.info(m), grouped.info(m)
        assert ia["status"] == ib["status"], m
        for q in range(2):
            for key in ("cycles", "arnoldi_steps", "converged", "residual_norm"):
                assert ia["solves"][q][key] == ib["solves"][q][key], (m, q, key)
        cycles.append(ib["solves"][0]["cycles"])
    assert cycles[2] <= 1  # the member with maxiter 1 stopped after at most one cycle
    assert grouped.info(0)["status"] == 0 and grouped.info(1)["status"] == 0


def test_graph_reports_unconverged_solves():
    from suetes_b200 import PingPong
    st, ds0, bc = _member(16, 12, torch.float64, tol=1e-14, maxiter=1)
    ref, infos = _eager(st, ds0, bc, 2)
    assert infos[-1]["status"] == 1  # SISL_NOT_CONVERGED
    pp = PingPong([(st, ds0, bc)])
    pp.step()
    gi = pp.info(0)
    assert gi["status"] == 1
    assert gi["solves"][0]["cycles"] == 1 and not gi["solves"][0]["converged"]
    for k in FIELDS:
        assert torch.equal(pp.current()[0].t[k], ref.t[k]), k


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_every_launch_shape_gives_identical_results(dtype):
    """The autotuner's candidates (stencil blocks, column tiles) change only
    the launch shape: forward and transposed operators are bitwise equal."""
    from suetes_b200 import SemiImplicitSolver3D, VerticalPreconditioner
    st, ds0, bc = _member(37, 13, dtype)
    ph = st.physics
    bg = ph.precompute_bg(ph.bg_state_ref())
    sol = SemiImplicitSolver3D(ph, st.dt, alpha=st.alpha)
    core = sol._core(dtype, bg)
    pm = VerticalPreconditioner(ph, st.dt, alpha=st.alpha)
    pm.precompute_banded(bg)
    g = ph.grid
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = {k: torch.randn(g.shape_of(l), generator=gen, device="cuda", dtype=dtype)
         for k, l in (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("eta_dot", "w"))}
    ops = lambda: [sol.matvec_scaled(x, bg), sol.matvec_scaled(x, bg, transpose=True), pm(x), pm.transpose(x)]
    core.set_tuning()  # all knobs at variant 0
    ref = ops()
    for knob, n in (("matvec_block", 9), ("matvec_t_block", 4), ("precond_tile", 8), ("precond_t_tile", 5)):
        for v in range(1, n):
            core.set_tuning(**{knob: v})
            out = ops()
            for a, b in zip(out, ref):
                for k in a:
                    assert torch.equal(a[k], b[k]), (knob, v, k)
    choice = core.autotune()
    assert 0 <= choice["matvec_block"] < 9 and 0 <= choice["precond_tile"] < 8
    assert all(t > 0 for t in choice["us"])
    assert core.tuning()["matvec_block"] == choice["matvec_block"]
    core.set_tuning()


@pytest.mark.parametrize("dtype", [torch.float32])
def test_integrate_graph_equals_eager(dtype):
    """SISLStepper3D.integrate replays captured graphs for 4+ steps: the
    state it returns equals the eager integration bit for bit."""
    from suetes_b200.workloads import mountain_wave
    st, s0, bc = mountain_wave(24, 16, 12, dtype=dtype, device="cuda", solver_tol=1e-7)
    a = st.integrate(dict(s0), 0.0, 5, None, bc, graph=True)
    b = st.integrate(dict(s0), 0.0, 5, None, bc, graph=False)
    for k in ("u", "v", "w", "eta_dot", "pi", "th_v", "rho"):
        assert torch.equal(a[k], b[k]), k
