"""Manufactured explicit tendencies (verification/equation_tendency_convergence.py),
shared by the oracle test (CPU) and the CUDA test.

A smooth trigonometric state on a 2000 x 2000 x 10 km oblique-stereographic
box centred at 60N 30E (map factors, their gradients and Coriolis active,
g = 0, theta_bg = 300 + 0.01 z, pi_bg = 1, constant rho_bg): the discrete
explicit tendencies approach the analytic ones at second order in the grid
spacing (:200-246).  The analytic derivatives are written out here instead
of taken by automatic differentiation."""

import math

import torch

R_E, OMEGA = 6371229.0, 7.2921e-5
CP, CVD, RD, P0 = 1004.0, 717.0, 287.0, 100000.0
LX, LY, LZ = 2000000.0, 2000000.0, 10000.0
TH0 = 300.0
C = {"g": 0.0, "cp": CP, "cvd": CVD, "Rd": RD, "p0": P0}
RHO0 = P0 / (RD * TH0)
kx, ky, kz = 2.0 * math.pi / LX, 2.0 * math.pi / LY, math.pi / LZ

# the manufactured state (:29-51)
u_f = lambda x, y, z: 10.0 * torch.sin(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
v_f = lambda x, y, z: 15.0 * torch.cos(kx * x) * torch.sin(ky * y) * torch.sin(kz * z)
w_f = lambda x, y, z: 1.0 * torch.sin(kx * x) * torch.cos(ky * y) * torch.cos(kz * z)
pip_f = lambda x, y, z: 0.01 * torch.sin(kx * x) * torch.sin(ky * y) * torch.sin(kz * z)
thp_f = lambda x, y, z: 5.0 * torch.cos(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
thbg_f = lambda z: TH0 + 0.01 * z


def _m(x, y):
    return 1.0 + (x ** 2 + y ** 2) / (4.0 * R_E ** 2)


def analytic(grid, x, y, z, name):
    """The analytic tendency `name` at points (x, y, z) (:55-137)."""
    m = _m(x, y)
    dmdx, dmdy = x / (2.0 * R_E ** 2), y / (2.0 * R_E ** 2)
    thv = thbg_f(z) + thp_f(x, y, z)
    if name in ("u", "v"):
        lat = grid.proj.get_lat_lon(x, y)[0]
        f = 2.0 * OMEGA * torch.sin(torch.deg2rad(lat))
        u, v = u_f(x, y, z), v_f(x, y, z)
        metric = v * dmdx - u * dmdy
        if name == "u":
            dpdx = 0.01 * kx * torch.cos(kx * x) * torch.sin(ky * y) * torch.sin(kz * z)
            return -CP * thv * m * dpdx + f * v + metric * v
        dpdy = 0.01 * ky * torch.sin(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
        return -CP * thv * m * dpdy - f * u - metric * u
    if name == "w":
        dpdz = 0.01 * kz * torch.sin(kx * x) * torch.sin(ky * y) * torch.cos(kz * z)
        return -CP * thv * dpdz
    if name == "th_v":
        return -w_f(x, y, z) * 0.01
    # pi: -C_pi (m^2 (d/dx(rho th u / m) + d/dy(rho th v / m)) + d/dz(rho th w))
    th = thbg_f(z)
    u, v = u_f(x, y, z), v_f(x, y, z)
    dudx = 10.0 * kx * torch.cos(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
    dvdy = 15.0 * ky * torch.cos(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
    dfx = RHO0 * th * (dudx / m - u * dmdx / m ** 2)
    dfy = RHO0 * th * (dvdy / m - v * dmdy / m ** 2)
    dwdz = -1.0 * kz * torch.sin(kx * x) * torch.cos(ky * y) * torch.sin(kz * z)
    dfz = RHO0 * (0.01 * w_f(x, y, z) + th * dwdz)
    cpi = (RD / CVD) * 1.0 / (RHO0 * th)
    return -cpi * (m ** 2 * (dfx + dfy) + dfz)


def _mesh(a, b, c):
    return torch.meshgrid(a.double().cpu(), b.double().cpu(), c.double().cpu(), indexing="ij")


def errors(pkg, n, device=None, faces="analytic"):
    """RMS errors of the five explicit tendencies on an n^3 grid, two points
    in from every boundary (:139-197).  The oracle takes theta' at the faces
    as the reference does (faces="analytic") or as the face averages of the
    mass-point values (faces="averaged", what the CUDA kernel forms)."""
    if pkg == "oracle":
        from oracle.grid import RegionalGrid3D
        from oracle.ops import CGridOperator3D
        from oracle.euler import Euler3D
        kw = {}
    else:
        from suetes_b200 import RegionalGrid3D, CGridOperator3D, Euler3D
        kw = {"device": device}
    g = RegionalGrid3D(n, n, n, LX / n, LY / n, LZ / n, 60.0, 30.0, **kw)
    op = CGridOperator3D(g)
    eu = Euler3D(g, op, C, dt=1.0, N_bv=0.0, nu_h_factor=0.0, nu_div_factor=0.0)
    pts = {"u": _mesh(g.x_c, g.y_m, g.z_m), "v": _mesh(g.x_m, g.y_c, g.z_m), "w": _mesh(g.x_m, g.y_m, g.z_c),
           "m": _mesh(g.x_m, g.y_m, g.z_m)}
    dev = (lambda t: t) if pkg == "oracle" else (lambda t: t.to(device))
    sp = {"u": u_f(*pts["u"]), "v": v_f(*pts["v"]), "w": w_f(*pts["w"]), "pi": pip_f(*pts["m"])}
    sp["eta_dot"] = sp["w"] / g.dz_w_full.double().cpu()
    if pkg == "oracle" and faces == "analytic":  # the face values of theta' as the reference passes them
        sp.update(th_v_prime_u=thp_f(*pts["u"]), th_v_prime_v=thp_f(*pts["v"]), th_v_prime_w=thp_f(*pts["w"]))
    elif pkg == "oracle":
        tm = thp_f(*pts["m"])
        sp.update(th_v_prime_u=op.avg(tm, 0, "m", "u"), th_v_prime_v=op.avg(tm, 1, "m", "v"),
                  th_v_prime_w=op.avg(tm, 2, "m", "w"))
    else:  # the CUDA kernel averages the mass-point theta' to the faces itself
        sp["th_v_prime_m"] = thp_f(*pts["m"])
    sp = {k: dev(t) for k, t in sp.items()}
    zm = pts["m"][2]
    bg = eu.precompute_bg({"rho": dev(RHO0 + 0.0 * zm), "pi": dev(1.0 + 0.0 * zm), "th_v": dev(thbg_f(zm))})
    tend = eu.get_tendencies(sp, bg, is_explicit=True)
    sl = (slice(2, -2),) * 3
    out = {}
    for name, loc in (("u", "u"), ("v", "v"), ("w", "w"), ("pi", "m"), ("th_v", "m")):
        ana = analytic(g, *pts[loc], name)
        d = tend[name].detach().double().cpu()[sl] - ana[sl]
        out[name] = float(torch.sqrt(torch.mean(d ** 2)))
    return out


def rates(errs):
    """log2 of successive error ratios for the n, 2n, 4n family."""
    return {k: [math.log2(a[k] / b[k]) for a, b in zip(errs[:-1], errs[1:])] for k in errs[0]}
