"""The CPU oracle against the reference's known answers and invariants.

The reference ships no golden outputs for the unsplit hydro path; its only
known answer is the analytic Sod shock tube (Sod/shocktube.pro,
soderror.pro).  These tests pin the oracle's restatement to that solution
(convergence under refinement, wave positions) and to invariants the scheme
must keep: uniform states, x/y symmetry, exact conservation with periodic
boundaries, and agreement of the two block orders.
"""
import json
import os

import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import next_dt
from flash5_b200 import metrics as sfocu
from oracle import orc, sod_exact

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def evolve(o, unk, tmax=None, nsteps=None, dt_cap=None):
    _, dt, _ = o.compute_dt(unk)
    if dt_cap:
        dt = min(dt, dt_cap)
    t, dt_old, n = 0.0, dt, 0
    while True:
        if tmax is not None:
            if t >= tmax - 1e-14:
                break
            dt = min(dt, tmax - t)
        if nsteps is not None and n >= nsteps:
            break
        assert o.hydro(unk, t + dt, dt, dt_old) == 0
        t += dt
        n += 1
        _, dcfl, _ = o.compute_dt(unk)
        dt_old, dt = dt, next_dt(dcfl, dt)
    return t, n


def sod_run(nblk, tmax=0.2, axis=0, nb=8, **pkw):
    g = UniformGrid(2, (nb, nb), (nblk, 1) if axis == 0 else (1, nblk), bc="outflow")
    p = abi.default_params(**pkw)
    unk = setups.sod(g) if axis == 0 else setups.sod_axis(g, axis=axis)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    t, n = evolve(o, unk, tmax=tmax, dt_cap=1e-3)
    return g, unk, t


def test_shocktube_restatement_matches_golden():
    """The restated IDL secant solve (eps 1e-8) finds the mpmath root."""
    cases = json.load(open(os.path.join(GOLD, "sod_shocktube.json")))["cases"]
    for c in cases:
        p4 = sod_exact.post_shock_pressure(c["rhol"], c["pl"], c["rhor"], c["pr"], c["gamma"])
        assert abs(p4 / float(c["p4"]) - 1) < 1e-7, (c, p4)


@pytest.mark.parametrize("nblk", [8, 16, 32])
def test_sod_against_exact_solution(nblk):
    g, unk, t = sod_run(nblk)
    nx = nblk * 8
    x = (np.arange(nx) + 0.5) / nx
    rs, ps, vs = sod_exact.shocktube(1.0, 1.0, 0.0, 0.125, 0.1, 0.0, 1.4, 0.5, t, x)
    dens = g.to_global(unk, "dens")[0]
    pres = g.to_global(unk, "pres")[0]
    l1 = np.abs(dens - rs[None, :]).mean()
    # first-order convergence near discontinuities: error ~ 0.36/nx for Sod
    assert l1 < 0.4 / nx, (nx, l1)
    perr = sod_exact.sod_l1_pressure_error(pres.T, x, (np.arange(8) + 0.5) / 8, t)
    assert perr < 0.4 / nx, perr


def test_sod_convergence_rate():
    errs = []
    for nblk in (8, 16, 32):
        g, unk, t = sod_run(nblk)
        nx = nblk * 8
        x = (np.arange(nx) + 0.5) / nx
        rs, _, _ = sod_exact.shocktube(1.0, 1.0, 0.0, 0.125, 0.1, 0.0, 1.4, 0.5, t, x)
        errs.append(np.abs(g.to_global(unk, "dens")[0] - rs).mean())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 0.8), (errs, rates)


def test_sod_x_and_y_are_symmetric():
    gx, ux, _ = sod_run(8, tmax=0.05)
    gy, uy, _ = sod_run(8, tmax=0.05, axis=1)
    dx = gx.to_global(ux, "dens")[0]
    dy = gy.to_global(uy, "dens")[0].T
    assert np.array_equal(dx, dy)
    vy = gy.to_global(uy, "vely")[0].T
    vx = gx.to_global(ux, "velx")[0]
    assert np.array_equal(vx, vy)


@pytest.mark.parametrize("rs", [abi.RS_HLLC, abi.RS_EXACT])
@pytest.mark.parametrize("ndim", [2, 3])
def test_uniform_state_is_preserved(ndim, rs):
    nb = (8, 8, 8)[:ndim]
    g = UniformGrid(ndim, nb, (2,) * ndim, bc="periodic")
    p = abi.default_params(riemann_solver=rs)
    unk = setups.uniform(g, rho=1.3, v=(0.3, -0.2, 0.1), p=0.7)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    before = g.interior(unk).copy()
    evolve(o, unk, nsteps=3)
    after = g.interior(unk)
    for v in ("dens", "velx", "vely", "velz", "pres"):
        np.testing.assert_allclose(after[..., VAR[v]], before[..., VAR[v]], rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("rs", [abi.RS_HLLC, abi.RS_EXACT])
@pytest.mark.parametrize("ndim", [2, 3])
def test_periodic_conservation(ndim, rs):
    nb = (8, 8, 8)[:ndim]
    g = UniformGrid(ndim, nb, (2, 3, 2)[:ndim], bc="periodic")
    p = abi.default_params(gamma=5.0 / 3.0, riemann_solver=rs)
    unk = setups.kelvin_helmholtz(g)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    c0 = sfocu.conserved(g.interior(unk), VAR)
    tot0 = {k: c0[k].sum() for k in c0}
    evolve(o, unk, nsteps=4)
    c1 = sfocu.conserved(g.interior(unk), VAR)
    for k in ("dens", "xmom", "ymom", "ener"):
        scale = np.abs(c0[k]).sum()
        assert abs(c1[k].sum() - tot0[k]) <= 1e-13 * scale, (k, c1[k].sum() - tot0[k])


def test_block_order_does_not_matter():
    g1 = UniformGrid(2, (8, 8), (4, 4), bc="outflow")
    g2 = UniformGrid(2, (8, 8), (4, 4), bc="outflow", order="morton")
    p = abi.default_params()
    out = []
    for g in (g1, g2):
        unk = setups.sod(g, xangle=45.0)
        o = orc.Oracle(p, g)
        o.eos_init(unk)
        evolve(o, unk, nsteps=3)
        out.append(g.to_global(unk, "dens"))
    assert np.array_equal(out[0], out[1])


def test_block_list_updates_only_listed_blocks():
    g = UniformGrid(2, (8, 8), (3, 2), bc="outflow")
    p = abi.default_params()
    unk = setups.sod(g, xangle=45.0)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    full = unk.copy()
    _, dt, _ = o.compute_dt(unk)
    o.hydro(full, dt, dt, dt)
    part = unk.copy()
    o.hydro(part, dt, dt, dt, blocks=[1, 4])
    it_f, it_p, it_0 = g.interior(full), g.interior(part), g.interior(unk)
    for b in range(g.nblocks):
        ref = it_f[b] if b in (1, 4) else it_0[b]
        assert np.array_equal(it_p[b][..., VAR["dens"]], ref[..., VAR["dens"]])


def test_negative_pressure_input_reports_status():
    """A non-physical state (negative pressure) raises the status FLASH aborts on."""
    g = UniformGrid(2, (8, 8), (2, 2), bc="outflow")
    p = abi.default_params()
    unk = setups.uniform(g)
    it = g.interior(unk)
    it[0, 0, 3, 3, VAR["eint"]] = -1.0
    it[0, 0, 3, 3, VAR["ener"]] = -1.0
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    st = o.hydro(unk, 1e-3, 1e-3, 1e-3)
    assert st & abi.ERR_NEG_SOUNDSPEED


def test_exact_star_state_matches_golden():
    cases = json.load(open(os.path.join(GOLD, "riemann_star.json")))["cases"]
    for c in cases:
        st, ps, us, it = orc.star_state(c["dl"], c["ul"], c["pl"], c["dr"], c["ur"], c["pr"], c["gamma"])
        assert st == 0, (c, st)
        assert abs(ps / float(c["pstar"]) - 1) < 1e-11, (c, ps)
        assert abs(us - float(c["ustar"])) < 1e-10 * max(1.0, abs(float(c["ustar"]))), (c, us)
    # the Sod p* from the shock-tube equation and from Toro's functions agree
    sod = json.load(open(os.path.join(GOLD, "sod_shocktube.json")))["cases"][0]
    assert abs(float(sod["p4"]) / float(cases[0]["pstar"]) - 1) < 1e-25


def test_exact_solver_sod_against_exact_solution():
    """The hydro step with exact-solver fluxes converges to the Sod solution
    at least as well as the HLLC bound."""
    nblk = 16
    g, unk, t = sod_run(nblk, riemann_solver=abi.RS_EXACT)
    nx = nblk * 8
    x = (np.arange(nx) + 0.5) / nx
    rs, _, _ = sod_exact.shocktube(1.0, 1.0, 0.0, 0.125, 0.1, 0.0, 1.4, 0.5, t, x)
    l1 = np.abs(g.to_global(unk, "dens")[0] - rs[None, :]).mean()
    assert l1 < 0.4 / nx, l1


def test_exact_flux_vacuum_generation():
    """Vacuum-generating data (Toro 4.6): symmetric expansion gives zero flux
    at x/t = 0; a one-sided case samples the left fan or state."""
    VL = np.array([1.0, -6.0, 0.0, 0.0, 0.4, 1.4, 1.4, 1.0])
    VR = np.array([1.0, 6.0, 0.0, 0.0, 0.4, 1.4, 1.4, 1.0])
    F, st, _ = orc.exact_flux(1, VL, VR, 1.4)
    assert st == 0 and np.all(F == 0.0), F
    # left state supersonic to the right: the left state itself
    VL = np.array([1.0, 3.0, 0.5, 0.0, 0.4, 1.4, 1.4, 1.0])
    VR = np.array([1.0, 12.0, 0.0, 0.0, 0.4, 1.4, 1.4, 1.0])
    F, st, _ = orc.exact_flux(1, VL, VR, 1.4)
    E = 0.4 / 0.4 + 0.5 * (9.0 + 0.25)
    np.testing.assert_allclose(F, [3.0, 9.0 + 0.4, 1.5, 0.0, (E + 0.4) * 3.0, 0.4], rtol=1e-14)
