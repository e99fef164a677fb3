"""Analytic Sod shock-tube solution -- TEST INFRASTRUCTURE ONLY.

A Python restatement of the reference's IDL known answer
Simulation/SimulationMain/Sod/shocktube.pro: the shock-tube equation
f(p4) (lines 15-33), the secant solve for the post-shock pressure
(lines 90-120), the post-shock state and wave positions (lines 122-165) and
the piecewise solution averaged over ``subsample`` points per cell
(lines 166-237); plus the L1 pressure error of Sod/soderror.pro.
"""
import numpy as np


def _f(p4, p1, p5, rho1, rho5, gamma):
    z = (p4 / p5 - 1.0)
    c1 = np.sqrt(gamma * p1 / rho1)
    c5 = np.sqrt(gamma * p5 / rho5)
    gm1 = gamma - 1.0
    gp1 = gamma + 1.0
    g2 = 2.0 * gamma
    fact = gm1 / g2 * (c5 / c1) * z / np.sqrt(1.0 + gp1 / g2 * z)
    fact = (1.0 - fact) ** (g2 / gm1)
    return p1 * fact - p4


def post_shock_pressure(rhol, pl, rhor, pr, gamma, itmax=20, eps=1e-8):
    if pl > pr:
        rho1, p1, rho5, p5 = rhol, pl, rhor, pr
    else:
        rho1, p1, rho5, p5 = rhor, pr, rhol, pl
    p40, p41 = p1, p5
    f0 = _f(p40, p1, p5, rho1, rho5, gamma)
    it, err = 1, 100.0
    p4 = p41
    while it < itmax and err > eps:
        f1 = _f(p41, p1, p5, rho1, rho5, gamma)
        p4 = p41 - (p41 - p40) * f1 / (f1 - f0)
        err = abs(p4 - p41) / p41
        p40, p41, f0 = p41, p4, f1
        it += 1
    return p4


def shocktube(rhol, pl, ul, rhor, pr, ur, gamma, xi, t, xpts, subsample=50):
    """Cell-averaged exact solution (rho, p, u) at the uniform mesh xpts."""
    xpts = np.asarray(xpts, dtype=np.float64)
    npts = len(xpts)
    nss = npts * subsample + 1
    dx = xpts[2] - xpts[1]
    xl = xpts[0] - 0.5 * dx
    xs = np.arange(nss) * (dx / subsample) + xl
    if pl > pr:
        rho1, p1, u1, rho5, p5, u5 = rhol, pl, ul, rhor, pr, ur
    else:
        rho1, p1, u1, rho5, p5, u5 = rhor, pr, ur, rhol, pl, ul
    p4 = post_shock_pressure(rhol, pl, rhor, pr, gamma)
    z = (p4 / p5 - 1.0)
    c5 = np.sqrt(gamma * p5 / rho5)
    gm1, gp1 = gamma - 1.0, gamma + 1.0
    gmfac1 = 0.5 * gm1 / gamma
    gmfac2 = 0.5 * gp1 / gamma
    fact = np.sqrt(1.0 + gmfac2 * z)
    u4 = c5 * z / (gamma * fact)
    rho4 = rho5 * (1.0 + gmfac2 * z) / (1.0 + gmfac1 * z)
    w = c5 * fact
    p3, u3 = p4, u4
    rho3 = rho1 * (p3 / p1) ** (1.0 / gamma)
    c1 = np.sqrt(gamma * p1 / rho1)
    c3 = np.sqrt(gamma * p3 / rho3)
    rho = np.empty(nss); p = np.empty(nss); u = np.empty(nss)
    if pl > pr:
        xsh, xcd, xft, xhd = xi + w * t, xi + u3 * t, xi + (u3 - c3) * t, xi - c1 * t
        for i, x in enumerate(xs):
            if x < xhd:
                rho[i], p[i], u[i] = rho1, p1, u1
            elif x < xft:
                u[i] = 2.0 / gp1 * (c1 + (x - xi) / t)
                f = 1.0 - 0.5 * gm1 * u[i] / c1
                rho[i] = rho1 * f ** (2.0 / gm1)
                p[i] = p1 * f ** (2.0 * gamma / gm1)
            elif x < xcd:
                rho[i], p[i], u[i] = rho3, p3, u3
            elif x < xsh:
                rho[i], p[i], u[i] = rho4, p4, u4
            else:
                rho[i], p[i], u[i] = rho5, p5, u5
    else:
        xsh, xcd, xft, xhd = xi - w * t, xi - u3 * t, xi - (u3 - c3) * t, xi + c1 * t
        for i, x in enumerate(xs):
            if x < xsh:
                rho[i], p[i], u[i] = rho5, p5, -u5
            elif x < xcd:
                rho[i], p[i], u[i] = rho4, p4, -u4
            elif x < xft:
                rho[i], p[i], u[i] = rho3, p3, -u3
            elif x < xhd:
                u[i] = -2.0 / gp1 * (c1 + (xi - x) / t)
                f = 1.0 + 0.5 * gm1 * u[i] / c1
                rho[i] = rho1 * f ** (2.0 / gm1)
                p[i] = p1 * f ** (2.0 * gamma / gm1)
            else:
                rho[i], p[i], u[i] = rho1, p1, -u1
    rs, ps, vs = np.empty(npts), np.empty(npts), np.empty(npts)
    for i in range(npts):
        sl = slice(subsample * i, subsample * (i + 1) + 1)
        rs[i], ps[i], vs[i] = rho[sl].mean(), p[sl].mean(), u[sl].mean()
    return rs, ps, vs


def sod_l1_pressure_error(comppres, x, y, t, rhol=1.0, pl=1.0, rhor=0.125, pr=0.1, gamma=1.4, xi=0.5):
    """soderror.pro without shock excision: sum |p - p_exact| dx dy."""
    _, psoln, _ = shocktube(rhol, pl, 0.0, rhor, pr, 0.0, gamma, xi, t, x)
    dp = comppres - psoln[:, None]
    dv = (x[2] - x[1]) * ((y[2] - y[1]) if len(y) > 2 else 1.0)
    return np.abs(dp).sum() * dv
