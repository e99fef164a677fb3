"""Hydro step on AMR hierarchies on the GPU vs the CPU oracle (marked gpu).

The device path (restriction, parent halos, leaf guard cells, one launch
per level and direction with the fine/coarse flux register) must give the
oracle's AMR step (oracle/flash_hy_oracle.c, PARAMESH-form restatement)
bit for bit on the FP64 path, in every leaf variable and in the time step
and its location; the mixed path stays within 1e-6 relative L1 and the
exact-solver path within the solver tolerance.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.amr import AmrGrid, indicator_refiner
from flash5_b200.grid import VAR
from flash5_b200.hydro import Hydro, next_dt
from oracle import orc
from tests.test_gpu_parity import conserved_l1

VARS = ("dens", "velx", "vely", "velz", "eint", "ener", "pres", "temp", "gamc", "game")


def ring(ndim, nb, nblk, max_level, bc, r2=0.06, w=0.004, **sk):
    """Hierarchy refined around a circle (sphere): leaves on several levels."""
    g = AmrGrid(ndim, (nb,) * ndim, (nblk,) * ndim, max_level, bc=bc, **sk)
    f = lambda X, Y, Z: 1.0 + 0.8 * np.tanh(((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.5) ** 2 * (ndim > 2) - r2) / w)
    g.refine_levels(indicator_refiner(g, f, 0.05))
    return g


def amr_case(name, nspecies=0, nmass_scalars=0, **pkw):
    sk = {"nspecies": nspecies, "nmass_scalars": nmass_scalars}
    if name == "kh2d_ring":
        g = ring(2, 8, 8, 3, "periodic", r2=0.02, w=0.002, **sk)
        u, p = setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    elif name == "quad2d_16":
        g = ring(2, 16, 6, 3, "outflow", r2=0.02, w=0.003, **sk)
        u, p = setups.four_quadrant(g), abi.default_params(**pkw)
    elif name == "sod2d_reflect":
        g = ring(2, 8, 8, 3, "reflecting", r2=0.01, w=0.002, **sk)
        u, p = setups.sod(g, xangle=30.0), abi.default_params(**pkw)
    elif name == "kh3d_ring":
        g = ring(3, 8, 2, 3, "periodic", **sk)
        u, p = setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    else:
        raise KeyError(name)
    return g, setups.add_species(g, u), p


def run_amr_pair(case, nsteps=4, **pkw):
    grid, unk0, params = amr_case(case, **pkw)
    return _run_amr(grid, unk0, params, nsteps)


def _run_amr(grid, unk0, params, nsteps):
    ref = unk0.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    h.upload(unk0)
    st, dt, loc = o.compute_dt(ref)
    steps = []
    t, dt_old = 0.0, dt
    for _ in range(nsteps):
        assert o.hydro(ref, t + dt, dt, dt_old) == 0
        h(t + dt, dt, dt_old)
        t += dt
        st, dto, loco = o.compute_dt(ref)
        dtg, locg = h.compute_dt()
        steps.append((dto, loco, dtg, locg))
        dt_old, dt = dt, next_dt(dto, dt)
    out = grid.new_unk()
    h.download(out)
    h.close()
    return grid, ref, out, steps


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_ring", "quad2d_16", "sod2d_reflect", "kh3d_ring"])
def test_amr_fp64_bitwise(case):
    grid, ref, out, steps = run_amr_pair(case)
    assert grid.max_used_level == 3
    for dto, loco, dtg, locg in steps:
        assert dtg == dto, (dtg, dto)
        assert tuple(locg) == tuple(loco), (locg, loco)
    leaves = grid.leaf_ids
    a, b = grid.interior(out)[leaves], grid.interior(ref)[leaves]
    for v in VARS:
        diff = np.abs(a[..., VAR[v]] - b[..., VAR[v]])
        assert np.array_equal(a[..., VAR[v]], b[..., VAR[v]]), (v, diff.max(), np.argwhere(diff > 0)[:4])
    # parents hold the restriction of the leaves
    par = np.nonzero(~grid.is_leaf)[0]
    for v in ("dens", "velx", "vely", "eint", "ener"):
        np.testing.assert_array_equal(grid.interior(out)[par][..., VAR[v]], grid.interior(ref)[par][..., VAR[v]])


def leaf_l1(grid, out, ref):
    class G:
        pass
    g = G()
    leaves = grid.leaf_ids
    g.interior = lambda u: grid.interior(u)[leaves]
    return conserved_l1(out, ref, g)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_ring", "quad2d_16", "kh3d_ring"])
def test_amr_mixed_close(case):
    grid, ref, out, _ = run_amr_pair(case, precision=abi.PREC_MIXED)
    for k, l1 in leaf_l1(grid, out, ref).items():
        assert l1 <= 1e-6, (k, l1)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["quad2d_16", "kh3d_ring"])
def test_amr_exact_solver(case):
    grid, ref, out, _ = run_amr_pair(case, riemann_solver=abi.RS_EXACT)
    for k, l1 in leaf_l1(grid, out, ref).items():
        assert l1 <= 1e-10, (k, l1)


@pytest.mark.gpu
def test_amr_block_list_is_refused():
    grid, unk, params = amr_case("kh2d_ring")
    h = Hydro(params, grid)
    from flash5_b200.hydro import HydroError
    with pytest.raises(HydroError):
        h.step_blocks([0], 1e-3, 1e-3, 1e-3)
    h.close()
