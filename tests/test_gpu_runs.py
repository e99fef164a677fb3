"""Runs of blocks in the mixed-precision direction kernels (marked gpu).

On a full uniform 3D grid of 8^3 blocks whose block counts divide by 4, the
mixed-precision direction kernels stage runs of four blocks that follow one
another along the sweep, a quarter of their cross-section per CTA, and the
last direction merges the quarters' CFL candidates per block (tuning
mx_runs = 4, the default there); with mx_runs = 1 a CTA takes one block.
Each cell and face is computed by the same source arithmetic either way,
but the two are separately compiled FMA-contracted kernels, as the
mx_threads candidates are: the time step locations must be equal, the time
steps and every UNK variable equal to rounding (1e-13 of each variable's
scale, floor 1).  The step over a block list (FLASH4's Hydro(blockCount,
blockList, ...), here listing every block) takes one block per CTA through
the same kernels as mx_runs = 1 and must match it bit for bit.  Cases: periodic
Kelvin-Helmholtz with HLLC, and a rotated 3D Sod problem with outflow and
reflecting boundaries (the slabs beyond them staged by the boundary rules)
with the exact solver and a trained learned guess (strong waves at the
shock, so the network is consulted).  Grids whose block counts do not
divide by 4 refuse mx_runs = 4.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro, HydroError, next_dt

VARS = ("dens", "velx", "vely", "velz", "eint", "ener", "pres", "temp", "gamc", "game")


def _kh():
    g = UniformGrid(3, (8, 8, 8), (8, 4, 4), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, precision=abi.PREC_MIXED), False


def _sod_exact_learned():
    g = UniformGrid(3, (8, 8, 8), (4, 4, 8), bc=["outflow", "outflow", "reflecting", "reflecting", "outflow",
                                                 "outflow"])
    p = abi.default_params(precision=abi.PREC_MIXED, riemann_solver=abi.RS_EXACT, learned_guess=1)
    return g, setups.sod(g, xangle=30.0, yangle=70.0), p, True


def _weights():
    from flash5_b200.riemann import ExactRiemann
    rs = ExactRiemann(0)
    try:
        rs.fit(rs.generate(7, 100_000), epochs=1, batch=4096)
        return rs.weights()
    finally:
        rs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", [_kh, _sod_exact_learned])
def test_runs_match_one_block_per_cta(case):
    grid, unk, params, learned = case()
    w = _weights() if learned else None
    runs, single, listed = Hydro(params, grid), Hydro(params, grid), Hydro(params, grid)
    try:
        assert runs.tuning["mx_runs"] == 4
        single.tuning = dict(single.tuning, mx_runs=1)
        for h in (runs, single, listed):
            if w is not None:
                h.set_guess_weights(w)
            h.upload(unk)
        every = list(range(grid.nblocks))
        dt, loc = runs.compute_dt()
        t, dt_old = 0.0, dt
        for _ in range(4):
            runs(t + dt, dt, dt_old)
            single(t + dt, dt, dt_old)
            listed.step_blocks(every, t + dt, dt, dt_old)
            t += dt
            d1, l1 = runs.compute_dt()
            d2, l2 = single.compute_dt()
            assert tuple(l1) == tuple(l2) and abs(d1 - d2) <= 1e-13 * d2, (d1, d2, l1, l2)
            dt_old, dt = dt, next_dt(d1, dt)
        # the run path was the one taken: the step's launches are the dt
        # store, k_sig, three direction kernels and the quarters' CFL merge
        runs(t + dt, dt, dt_old)
        single(t + dt, dt, dt_old)
        listed.step_blocks(every, t + dt, dt, dt_old)
        assert (runs.last_launch_count, single.last_launch_count) == (6, 5)
        a, b, c = grid.new_unk(), grid.new_unk(), grid.new_unk()
        runs.download(a)
        single.download(b)
        listed.download(c)
        for v in VARS:
            x, y, z = (grid.interior(u)[..., VAR[v]] for u in (a, b, c))
            lim = 1e-13 * max(float(np.abs(y).max()), 1.0)
            assert float(np.abs(x - y).max()) <= lim, (v, float(np.abs(x - y).max()))
            assert np.array_equal(y, z), (v, float(np.abs(y - z).max()))
    finally:
        runs.close()
        single.close()
        listed.close()


@pytest.mark.gpu
def test_runs_need_block_counts_divisible_by_four():
    g = UniformGrid(3, (8, 8, 8), (6, 4, 4), bc="periodic")
    h = Hydro(abi.default_params(gamma=5.0 / 3.0, precision=abi.PREC_MIXED), g)
    try:
        assert h.tuning["mx_runs"] == 1
        with pytest.raises(HydroError):
            h.tuning = dict(h.tuning, mx_runs=4)
    finally:
        h.close()
