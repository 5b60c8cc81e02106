"""The native reverse sweep of the step (``sisl_step_vjp``) and of the
explicit tendencies (``sisl_explicit_tendencies_vjp``) against autograd
through ``DifferentiableStep``, which the oracle pins (test_gpu_adjoint.py):
float64 agreement to round-off and the solver tolerance, for every output
cotangent (history and rho included), first and later steps, open and
periodic axes, the limiter and the lateral relaxation."""

import pytest
import torch

from _cases import build, mountain, rel_l2, to_cuda

pytestmark = pytest.mark.gpu

OUT_KEYS = ("u", "v", "w", "eta_dot", "pi_p", "th_p", "rho", "u_prev", "v_prev", "w_prev", "eta_dot_prev",
            "tend_th_prev")
IN_KEYS = ("u", "v", "w", "eta_dot", "pi_p", "th_p")


def _setup(periodic=(), limiter=False, dtype=torch.float64, nx=12, ny=10, nz=9):
    from suetes_b200 import SISLStepper3D as PSt
    from test_gpu_adjoint import _bubble
    kw = dict(dt=10.0, N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1, damp_height=4000.0, max_damp=0.5,
              lat=45.0, periodic=periodic)
    o = build("oracle", nx, ny, nz, 500.0, 500.0, 500.0, h=mountain, **kw)
    p = build("cuda", nx, ny, nz, 500.0, 500.0, 500.0, h=mountain, device="cuda", **kw)
    tol = 1e-13 if dtype == torch.float64 else 1e-7
    st = PSt(p[2], 10.0, alpha=0.55, use_limiter=limiter, solver_tol=tol, solver_maxiter=80, solver_restart=40)
    st.implicit_solver.transpose_tol = tol
    s0 = to_cuda(_bubble(o[2], o[0]))
    if dtype != torch.float64:
        s0 = {k: v.to(dtype) if torch.is_tensor(v) else v for k, v in s0.items()}
    return st, s0, p


def _cotangents(ds, seed):
    gen = torch.Generator().manual_seed(seed)
    return {k: torch.randn(tuple(t.shape), generator=gen, dtype=torch.float64).to(t.device, t.dtype)
            for k, t in ds.t.items() if k in OUT_KEYS}


def _autograd_vjp(st, ds, rec, cot, relax):
    from suetes_b200.adjoint import DifferentiableStep
    dstep = DifferentiableStep(st, ds.core.dtype)
    before = {k: v.detach().clone().requires_grad_(True) for k, v in ds.t.items()}
    with torch.enable_grad():
        out = dstep(dict(before, is_first_step=ds.is_first_step), relax=relax, recorded=rec)
        outs, grads = [], []
        for k, g in cot.items():
            if k in out and torch.is_tensor(out[k]) and out[k].requires_grad:
                outs.append(out[k])
                grads.append(g)
        gs = torch.autograd.grad(outs, [before[k] for k in IN_KEYS], grads, allow_unused=True)
    return {k: (g if g is not None else torch.zeros_like(before[k])) for k, g in zip(IN_KEYS, gs)}


@pytest.mark.parametrize("relaxed", [False, True])
@pytest.mark.parametrize("periodic,limiter", [((), False), ((), True), ((0,), False), ((0, 1), True)])
def test_native_step_vjp_matches_autograd(periodic, limiter, relaxed):
    from suetes_b200 import x_relaxation
    from suetes_b200.adjoint import _taped_step, step_vjp
    st, s0, p = _setup(periodic, limiter)
    relax = x_relaxation(p[0], 1000.0, 3.0) if relaxed and 0 not in periodic else None
    ds = st.to_device_state(s0)
    for n in range(2):  # the first step (no extrapolation) and a later one
        nxt, rec = _taped_step(st, ds, relax)
        cot = _cotangents(nxt, 100 + n)
        g_nat = step_vjp(st, ds, rec, cot, relax=relax)
        g_ref = _autograd_vjp(st, ds, rec, cot, relax)
        for k in IN_KEYS:
            err = rel_l2(g_nat[k], g_ref[k])
            assert err < 1e-8, (n, k, err)  # transposed solves at tol 1e-13 on rhs equal to rounding
        ds = nxt


def test_native_step_vjp_partial_cotangents():
    """Missing output cotangents are zero; rho and history members of in_bar are zeroed."""
    import ctypes
    from suetes_b200 import _lib
    from suetes_b200.adjoint import _taped_step, step_vjp
    st, s0, p = _setup()
    ds = st.to_device_state(s0)
    nxt, rec = _taped_step(st, ds, None)
    cot = {"w": _cotangents(nxt, 3)["w"]}
    g_nat = step_vjp(st, ds, rec, cot)
    g_ref = _autograd_vjp(st, ds, rec, cot, None)
    for k in IN_KEYS:
        assert rel_l2(g_nat[k], g_ref[k]) < 1e-8, k
    # in_bar members with no cotangent are written as zeros
    core = ds.core
    junk = {k: torch.full(tuple(t.shape), 7.0, dtype=t.dtype, device=t.device) for k, t in ds.t.items()}
    ib, ob = _lib.SislState(), _lib.SislState()
    for k, t in junk.items():
        setattr(ib, k, t.data_ptr())
    ws, n = core.workspace(_lib.WS_STEP_VJP)
    sin = ds.c_struct()
    rc = core.lib.sisl_step_vjp(core.handle, ctypes.byref(sin), _lib.ptrs(rec[0] + rec[1], 10), None,
                                ctypes.byref(ob), ctypes.byref(ib), ws.data_ptr(), n, core.stream, None)
    assert rc == 0
    torch.cuda.synchronize()
    for k in junk:
        assert float(junk[k].abs().max()) == 0.0, k


def test_native_step_vjp_float32_close_to_float64():
    from suetes_b200.adjoint import _taped_step, step_vjp
    res = {}
    for dt_ in (torch.float64, torch.float32):
        st, s0, p = _setup(dtype=dt_)
        ds = st.to_device_state(s0)
        nxt, rec = _taped_step(st, ds, None)
        ds2, rec2 = _taped_step(st, nxt, None)
        cot = {k: v.to(dt_) for k, v in _cotangents(ds2, 11).items()}
        res[dt_] = step_vjp(st, nxt, rec2, cot)
    for k in IN_KEYS:
        err = rel_l2(res[torch.float32][k].double(), res[torch.float64][k])
        assert err < 1e-4, (k, err)


@pytest.mark.parametrize("periodic", [(), (0,), (0, 1)])
def test_explicit_tendencies_vjp_matches_autograd(periodic):
    from suetes_b200.adjoint import DifferentiableStep
    st, s0, p = _setup(periodic)
    ds = st.to_device_state(s0)
    ph = st.physics
    dstep = DifferentiableStep(st, torch.float64)
    leaves = {k: ds.t[k].detach().clone().requires_grad_(True) for k in ("u", "v", "w", "eta_dot", "pi_p", "th_p")}
    gen = torch.Generator().manual_seed(21)
    R = lambda t: torch.randn(tuple(t.shape), generator=gen, dtype=torch.float64).to(t.device)
    with torch.enable_grad():
        sp = {"u": leaves["u"], "v": leaves["v"], "w": leaves["w"], "pi": leaves["pi_p"],
              "eta_dot": leaves["eta_dot"]}
        tn = dstep.tendencies(sp, leaves["th_p"])
        nl = dstep.nonlinear_pi(sp, leaves["th_p"])
        tb = {"u": R(tn["u"]), "v": R(tn["v"]), "w": R(tn["w"]), "pi": R(tn["pi"]), "th_v": R(tn["th_v"]),
              "nl_pi": R(nl)}
        pb = {"u": R(tn["u"]), "v": R(tn["v"]), "w": R(tn["w"]), "th_v": R(tn["th_v"])}
        J = sum((tb[k] * tn[k]).sum() for k in ("u", "v", "w", "pi", "th_v")) + (tb["nl_pi"] * nl).sum()
        J = J + sum((pb[k] * tn["phys_diff_" + k]).sum() for k in ("u", "v", "w", "th_v"))
        gs = dict(zip(leaves, torch.autograd.grad(J, list(leaves.values()))))
    bg = ph.precompute_bg(ph.bg_state_ref())
    g = ph.explicit_tendencies_vjp({"u": ds.t["u"], "v": ds.t["v"], "w": ds.t["w"], "pi": ds.t["pi_p"],
                                    "eta_dot": ds.t["eta_dot"]}, ds.t["th_p"], bg, tb, pb)
    for kn, kr in (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "pi_p"), ("eta_dot", "eta_dot"), ("th_p", "th_p")):
        err = rel_l2(g[kn], gs[kr])
        assert err < 1e-11, (kn, err)


def test_ensemble_vjp_concurrent_matches_sequential():
    """Members driven concurrently (own stream and host thread each) give the
    gradients of the same members one after another.  Open boundaries only:
    on a periodic axis the transposed system is inconsistent and its GMRES
    runs to maxiter, so its result follows the atomic summation order of
    the scatter kernels, concurrent or not."""
    from suetes_b200.adjoint import ensemble_trajectory_vjp, trajectory_vjp
    members = []
    for periodic, nx in (((), 12), ((), 10), ((), 14)):
        st, s0, p = _setup(periodic, nx=nx)
        members.append((st, st.to_device_state(s0), None))

    def objective(m, n, s):
        return (s["w"] ** 2).sum() * (m + 1) if n == 2 else None

    conc = ensemble_trajectory_vjp(members, 2, objective, wrt=("th_p", "u"))
    for m, (st, ds, bc) in enumerate(members):
        J, g = trajectory_vjp(st, ds, 2, lambda n, s: objective(m, n, s), bc_fn=bc, wrt=("th_p", "u"))
        assert abs(float(conc[m][0]) - float(J)) <= 1e-12 * abs(float(J)), m
        for k in ("th_p", "u"):
            assert rel_l2(conc[m][1][k], g[k]) < 1e-10, (m, k)


def test_ensemble_vjp_graph_matches_eager():
    """The trajectory VJP replayed as CUDA graphs (taped forward and reverse
    sweep of every member per step) gives the eager sweeps' values and
    gradients, for an objective with terms at two steps, on two runs from
    different starts."""
    from suetes_b200.adjoint import EnsembleVJPGraph, ensemble_trajectory_vjp
    from suetes_b200.steppers import DeviceState
    members = []
    for nx in (12, 10):
        st, s0, p = _setup((), nx=nx)
        members.append((st, st.to_device_state(s0), None))

    def objective(m, n, s):
        w2 = (s["w"] ** 2).sum() * (m + 1)
        return w2 if n == 2 else (0.5 * (s["th_p"] ** 2).sum() if n == 1 else None)

    graph = EnsembleVJPGraph(members, 2)
    for trial in range(2):
        starts = []
        for st, ds, bc in members:
            t = {k: v.clone() for k, v in ds.t.items()}
            t["th_p"] = t["th_p"] * (1.0 + 0.1 * trial)
            starts.append(DeviceState(ds.core, t, ds.is_first_step))
        got = graph.run(starts, objective, wrt=("th_p", "u", "w"))
        ref = ensemble_trajectory_vjp([(st, s, bc) for (st, _, bc), s in zip(members, starts)], 2, objective,
                                      wrt=("th_p", "u", "w"))
        for m in range(len(members)):
            assert abs(float(got[m][0]) - float(ref[m][0])) <= 1e-12 * abs(float(ref[m][0])), (trial, m)
            for k in ("th_p", "u", "w"):
                assert rel_l2(got[m][1][k], ref[m][1][k]) < 1e-10, (trial, m, k)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_grouped_ensemble_vjp_graph_equals_branches(dtype):
    """Grouped solves in both graphs of the ensemble VJP (the taped forward
    and the reverse sweep: one GMRES on A, then on A^T, over all members per
    solve) give every member's value and gradient the same bits as the
    graphs of per-member branches."""
    from suetes_b200.adjoint import EnsembleVJPGraph
    members = []
    for nx, ny, nz in ((12, 10, 9), (16, 12, 10), (10, 14, 8)):
        st, s0, p = _setup((), dtype=dtype, nx=nx, ny=ny, nz=nz)
        members.append((st, st.to_device_state(s0), None))

    def objective(m, n, s):
        return (s["w"] ** 2).sum() * (m + 1) if n == 2 else None

    branch = EnsembleVJPGraph(members, 2)
    grouped = EnsembleVJPGraph(members, 2, grouped=True)
    starts = [ds for _, ds, _ in members]
    ra = branch.run(starts, objective, wrt=("th_p", "u", "w"))
    rb = grouped.run(starts, objective, wrt=("th_p", "u", "w"))
    for m in range(len(members)):
        assert float(ra[m][0]) == float(rb[m][0]), m
        for k in ("th_p", "u", "w"):
            assert torch.equal(ra[m][1][k], rb[m][1][k]), (m, k)
        for q in range(2):
            a, b = branch.rev[0].info(m)["solves"][q], grouped.rev[0].info(m)["solves"][q]
            assert a["cycles"] == b["cycles"] and a["converged"] == b["converged"], (m, q)


@pytest.mark.parametrize("limiter", [False, True])
def test_float32_step_vjp_is_bitwise_repeatable(limiter):
    """Every scatter of the reverse sweep sums in fixed point (the tricubic
    VJPs and the explicit and corrector stencil transposes), the Laplacian
    transposes are gathers and the transposed solves reduce in a fixed
    order: three sweeps of the same float32 step give the same bits."""
    from suetes_b200 import x_relaxation
    from suetes_b200.adjoint import _taped_step, step_vjp
    st, s0, p = _setup((), limiter, dtype=torch.float32, nx=40, ny=32, nz=16)
    relax = x_relaxation(p[0], 2000.0, 3.0)
    ds = st.to_device_state(s0)
    ds, _ = _taped_step(st, ds, relax)  # a later step: extrapolated trajectories
    nxt, rec = _taped_step(st, ds, relax)
    cot = _cotangents(nxt, 7)
    runs = [step_vjp(st, ds, rec, cot, relax=relax) for _ in range(3)]
    for r in runs[1:]:
        for k in IN_KEYS:
            assert torch.equal(r[k], runs[0][k]), k
