"""VJP of the flux-form semi-Lagrangian transport (``sisl_ffsl_advect_vjp``,
``sisl_ffsl_lines_vjp``) against autograd through the float64 oracle, which
restates jnp.clip's tie rule (steppers.py:586-591): a departure interface
exactly on a wall passes half its cotangent."""

import pytest
import torch

from _cases import build, mountain, rel_l2, to_cuda

pytestmark = pytest.mark.gpu


def _state(nx, ny, nz, seed, walls_at_rest=True):
    gen = torch.Generator().manual_seed(seed)
    st = {"u": 10.0 + 8.0 * torch.rand(nx + 1, ny, nz, generator=gen, dtype=torch.float64),
          "v": -4.0 + 6.0 * torch.rand(nx, ny + 1, nz, generator=gen, dtype=torch.float64),
          "eta_dot": 4e-3 * (torch.rand(nx, ny, nz + 1, generator=gen, dtype=torch.float64) - 0.5)}
    if walls_at_rest:  # exact clip ties on the walls
        st["u"][0] = 0.0
        st["u"][-1] = 0.0
        st["v"][:, 0] = 0.0
        st["v"][:, -1] = 0.0
    st["eta_dot"][:, :, 0] = 0.0
    st["eta_dot"][:, :, -1] = 0.0
    rho = 1.0 + 0.1 * torch.rand(nx, ny, nz, generator=gen, dtype=torch.float64)
    return rho, st


@pytest.mark.parametrize("periodic", [(), (0,), (0, 1)])
def test_ffsl_advect_vjp_matches_oracle(periodic):
    from oracle.steppers import FluxFormAdvector as OF
    from suetes_b200 import FluxFormAdvector as PF
    nx, ny, nz, dt = 13, 11, 9, 150.0
    kw = dict(h=mountain, periodic=periodic, dt=dt, N_bv=0.01)
    og, _, oph = build("oracle", nx, ny, nz, 1000.0, 1000.0, 500.0, **kw)
    pg, _, pph = build("cuda", nx, ny, nz, 1000.0, 1000.0, 500.0, device="cuda", **kw)
    rho, st = _state(nx, ny, nz, 4, walls_at_rest=not periodic)
    gen = torch.Generator().manual_seed(9)
    wb = torch.randn(nx, ny, nz, generator=gen, dtype=torch.float64)
    leaves = {"rho": rho.clone().requires_grad_(True)}
    leaves.update({k: v.clone().requires_grad_(True) for k, v in st.items()})
    bgo = oph.precompute_bg(oph.bg_state_ref())
    out = OF(og, dt, periodic_axes=periodic).advect_3d_split(leaves["rho"], leaves, bgo)
    g = dict(zip(leaves, torch.autograd.grad((wb * out).sum(), list(leaves.values()))))
    adv = PF(pg, dt, periodic_axes=periodic, physics=pph)
    bgp = pph.precompute_bg(pph.bg_state_ref())
    gp = adv.advect_3d_split_vjp(rho.cuda(), to_cuda(st), bgp, wb.cuda())
    assert rel_l2(gp["field"], g["rho"]) < 1e-12, rel_l2(gp["field"], g["rho"])
    for k in ("u", "v", "eta_dot"):
        assert rel_l2(gp[k], g[k]) < 1e-11, (k, rel_l2(gp[k], g[k]))


@pytest.mark.parametrize("periodic", [False, True])
def test_ffsl_lines_vjp_matches_oracle(periodic):
    from oracle.steppers import FluxFormAdvector as OF
    from suetes_b200 import FluxFormAdvector as PF, RegionalGrid3D
    N, L = 17, 40
    gen = torch.Generator().manual_seed(2)
    s = torch.rand(L, N, generator=gen, dtype=torch.float64)
    c = 6.0 * (torch.rand(L, N + 1, generator=gen, dtype=torch.float64) - 0.5)
    c[:10] = torch.round(c[:10])  # integer departure points (w = 0) and, on open lines, exact clip ties
    c[10:12, 0] = 0.0
    c[10:12, -1] = 0.0
    ob = torch.randn(L, N, generator=gen, dtype=torch.float64)
    so, co = s.clone().requires_grad_(True), c.clone().requires_grad_(True)
    from oracle.grid import RegionalGrid3D as OG
    out = OF(OG(4, 4, 4, 1.0, 1.0, 1.0, 0.0, 0.0), 1.0)._advect_last(so, co, periodic)
    gs, gc = torch.autograd.grad((ob * out).sum(), [so, co])
    adv = PF(RegionalGrid3D(4, 4, 4, 1.0, 1.0, 1.0, 0.0, 0.0, device="cuda"), 1.0)
    ps, pc = adv.advect_1d_vjp(s.cuda(), c.cuda(), ob.cuda(), periodic=periodic)
    assert rel_l2(ps, gs) < 1e-13, rel_l2(ps, gs)
    assert rel_l2(pc, gc) < 1e-13, rel_l2(pc, gc)


def test_ffsl_advect_vjp_float32_close_to_float64():
    from suetes_b200 import FluxFormAdvector as PF
    nx, ny, nz, dt = 16, 12, 10, 150.0
    res = {}
    rho, st = _state(nx, ny, nz, 6)
    wb = torch.randn(nx, ny, nz, generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    for dtp in (torch.float64, torch.float32):
        pg, _, pph = build("cuda", nx, ny, nz, 1000.0, 1000.0, 500.0, h=mountain, device="cuda", dt=dt, N_bv=0.01)
        adv = PF(pg, dt, physics=pph)
        bgp = pph.precompute_bg(pph.bg_state_ref())
        res[dtp] = adv.advect_3d_split_vjp(rho.cuda().to(dtp), to_cuda(st, dtp), bgp, wb.cuda().to(dtp))
    for k in ("field", "u", "v", "eta_dot"):
        err = rel_l2(res[torch.float32][k].double(), res[torch.float64][k])
        assert err < 1e-5, (k, err)
