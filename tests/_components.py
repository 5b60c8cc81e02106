"""The reference's component convergence units 2 and 5-8
(verification/sisl_component_convergence.py:95-145, :266-449) on the oracle:
C-grid operators, explicit tendencies, the implicit linear operator, the
semi-Lagrangian advection and the flux-form advection, each on 16^3, 32^3
and 64^3 grids against its analytic counterpart.  The analytic derivatives
are written out instead of taken by automatic differentiation."""

import math

import torch

G, CP, CVD, RD, P0 = 9.81, 1004.0, 717.0, 287.0, 100000.0
LX, LY, LZ = 2000000.0, 2000000.0, 10000.0
R_E = 6371229.0


def _mesh(a, b, c):
    return torch.meshgrid(a, b, c, indexing="ij")


def _masked_rms(a, b, mask):  # compute_safe_err (:41-43)
    return float(torch.sqrt(torch.sum((a - b) ** 2 * mask) / torch.sum(mask)))


def unit2_operators(n):
    """diff m->u and avg m->u of a sine field on a 10 km Cartesian cube (:95-145)."""
    from oracle.grid import RegionalGrid3D
    from oracle.ops import CGridOperator3D
    L = 10000.0
    g = RegionalGrid3D(n, n, n, L / n, L / n, L / n, 0.0, 0.0)
    for k in g.m_factors:
        g.m_factors[k] = torch.ones_like(g.m_factors[k])
    op = CGridOperator3D(g)
    f = lambda x, y, z: torch.sin(2 * math.pi * x / L) * torch.cos(2 * math.pi * y / L) * torch.sin(2 * math.pi * z / L)
    X, Y, Z = _mesh(g.x_m, g.y_m, g.z_m)
    Xu, Yu, Zu = _mesh(g.x_c, g.y_m, g.z_m)
    fm = f(X, Y, Z)
    dfx = (2 * math.pi / L) * torch.cos(2 * math.pi * Xu / L) * torch.cos(2 * math.pi * Yu / L) * torch.sin(2 * math.pi * Zu / L)
    m = n // 4
    sl = (slice(m, -m),) * 3
    e_diff = float(torch.sqrt(torch.mean((op.diff(fm, 0, "m", "u")[sl] - dfx[sl]) ** 2)))
    e_avg = float(torch.sqrt(torch.mean((op.avg(fm, 0, "m", "u")[sl] - f(Xu, Yu, Zu)[sl]) ** 2)))
    return {"diff": e_diff, "avg": e_avg}


# units 5-7: the smooth state of :272-283 (sin^2 bumps), stratified background
TH0, NBV = 300.0, 0.01
_bump = lambda x, y, z: torch.sin(2 * math.pi * x / LX) ** 2 * torch.sin(2 * math.pi * y / LY) ** 2 * torch.sin(math.pi * z / LZ) ** 2


def _dbump(x, y, z, axis):
    sx, sy, sz = torch.sin(2 * math.pi * x / LX), torch.sin(2 * math.pi * y / LY), torch.sin(math.pi * z / LZ)
    cx, cy, cz = torch.cos(2 * math.pi * x / LX), torch.cos(2 * math.pi * y / LY), torch.cos(math.pi * z / LZ)
    if axis == 0:
        return 2 * sx * cx * (2 * math.pi / LX) * sy ** 2 * sz ** 2
    if axis == 1:
        return sx ** 2 * 2 * sy * cy * (2 * math.pi / LY) * sz ** 2
    return sx ** 2 * sy ** 2 * 2 * sz * cz * (math.pi / LZ)


th_bg_f = lambda z: TH0 * torch.exp((NBV ** 2 / G) * z)
pi_bg_f = lambda z: 1.0 + (G ** 2 / (CP * TH0 * NBV ** 2)) * (torch.exp(-NBV ** 2 * z / G) - 1.0)
rho_bg_f = lambda z: P0 / (RD * th_bg_f(z)) * pi_bg_f(z) ** (CVD / RD)


def units5_7(n, dt=60.0, alpha=0.55):
    """Explicit u/w tendencies, linear-operator u/w tendencies and the
    semi-Lagrangian advection of theta' at 60N (:266-404)."""
    from oracle.grid import RegionalGrid3D
    from oracle.ops import CGridOperator3D
    from oracle.euler import Euler3D
    from oracle.steppers import SemiLagrangianAdvector3D
    g = RegionalGrid3D(n, n, n, LX / n, LY / n, LZ / n, 60.0, 30.0)
    op = CGridOperator3D(g)
    ph = Euler3D(g, op, {"g": G, "cp": CP, "cvd": CVD, "Rd": RD, "p0": P0}, dt=dt, N_bv=NBV)
    adv = SemiLagrangianAdvector3D(g, ph, dt)
    Xu, Yu, Zu = _mesh(g.x_c, g.y_m, g.z_m)
    Xv, Yv, Zv = _mesh(g.x_m, g.y_c, g.z_m)
    Xw, Yw, Zw = _mesh(g.x_m, g.y_m, g.z_c)
    Xm, Ym, Zm = _mesh(g.x_m, g.y_m, g.z_m)
    bg = ph.precompute_bg({"rho": rho_bg_f(Zm), "pi": ph.pi_bg, "th_v": ph.theta_bg})
    sp = {"u": _bump(Xu, Yu, Zu), "v": _bump(Xv, Yv, Zv), "w": 0.1 * _bump(Xw, Yw, Zw), "pi": 0.01 * _bump(Xm, Ym, Zm),
          "th_v_prime_m": 5.0 * _bump(Xm, Ym, Zm)}
    sp["th_v_prime_w"] = op.avg(sp["th_v_prime_m"], 2, "m", "w")
    sp["th_v_prime_u"] = op.avg(sp["th_v_prime_m"], 0, "m", "u")
    sp["th_v_prime_v"] = op.avg(sp["th_v_prime_m"], 1, "m", "v")
    sp["eta_dot"] = sp["w"] / g.dz_w_full
    buf = 2000.0
    inner = lambda X, Y, Z: ((X.abs() < LX / 2 - 400000.0) & (Y.abs() < LY / 2 - 400000.0) & (Z >= buf)
                             & (Z <= LZ - buf)).double()
    mu, mw, mm = inner(Xu, Yu, Zu), inner(Xw, Yw, Zw), inner(Xm, Ym, Zm)
    f_u = g.f_u[..., None]

    def ana_u(explicit):
        m = 1.0 + (Xu ** 2 + Yu ** 2) / (4.0 * R_E ** 2)
        u, v = _bump(Xu, Yu, Zu), _bump(Xu, Yu, Zu)
        dpdx = 0.01 * _dbump(Xu, Yu, Zu, 0)
        if not explicit:
            return -CP * th_bg_f(Zu) * m * dpdx + f_u * v
        thv = th_bg_f(Zu) + 5.0 * _bump(Xu, Yu, Zu)
        metric = (v * Xu / (2.0 * R_E ** 2) - u * Yu / (2.0 * R_E ** 2)) * v
        return -CP * thv * m * dpdx + f_u * v + metric

    def ana_w(explicit):
        dpdz = 0.01 * _dbump(Xw, Yw, Zw, 2)
        if not explicit:
            return -CP * th_bg_f(Zw) * dpdz
        thp = 5.0 * _bump(Xw, Yw, Zw)
        return -CP * (th_bg_f(Zw) + thp) * dpdz + G * (thp / th_bg_f(Zw))

    te = ph.get_tendencies(sp, bg, is_explicit=True)
    L = ph.linear_operator(sp, bg, dt, alpha)
    tu = (sp["u"] - L["u"]) / (alpha * dt)
    tw = (sp["w"] - L["w"]) / (alpha * dt)
    coords = adv.compute_departure_indices(sp, loc="m", iterations=3)
    q = adv.advect_cubic(sp["th_v_prime_m"], coords, use_limiter=False)
    qa = 5.0 * _bump(Xm - dt * op.avg(sp["u"], 0, "u", "m"), Ym - dt * op.avg(sp["v"], 1, "v", "m"),
                     Zm - dt * op.avg(sp["w"], 2, "w", "m"))
    return {"exp_u": _masked_rms(te["u"], ana_u(True), mu), "exp_w": _masked_rms(te["w"], ana_w(True), mw),
            "imp_u": _masked_rms(tu, ana_u(False), mu), "imp_w": _masked_rms(tw, ana_w(False), mw),
            "adv_q": _masked_rms(q, qa, mm)}


def unit8_ffsl(n):
    """Flux-form advection of a sine density in a 10 m/s wind at Courant
    number 0.4 (:406-440)."""
    from oracle.grid import RegionalGrid3D
    from oracle.steppers import FluxFormAdvector
    L = 10000.0
    dx = L / n
    dt = (dx / 125.0) * 5.0
    g = RegionalGrid3D(n, n, n, dx, dx, dx, 0.0, 0.0)
    adv = FluxFormAdvector(g, dt)
    st = {"u": torch.ones(n + 1, n, n, dtype=torch.float64) * 10.0, "v": torch.zeros(n, n + 1, n, dtype=torch.float64),
          "eta_dot": torch.zeros(n, n, n + 1, dtype=torch.float64)}
    bgp = {"dz_m_full": torch.ones(n, n, n, dtype=torch.float64) * dx}
    X, Y, Z = _mesh(g.x_m, g.y_m, g.z_m)
    rho = torch.sin(2 * math.pi * X / L) + 2.0
    out = adv.advect_3d_split(rho, st, bgp)
    ex = torch.sin(2 * math.pi * (X - 10.0 * dt) / L) + 2.0
    m = n // 4
    sl = (slice(m, -m),) * 3
    return {"rho": float(torch.sqrt(torch.mean((out[sl] - ex[sl]) ** 2)))}


def rates(errs):
    return {k: [math.log2(a[k] / b[k]) for a, b in zip(errs[:-1], errs[1:])] for k in errs[0]}
