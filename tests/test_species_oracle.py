"""Species and mass scalars in the oracle (CPU): the restatement of
hy_fullSpecMsFluxHandling (PPM face values, upwind fluxes F_dens * X,
updateSpeciesMassScalar and the renormalisation of hy_unsplitUpdate.F90:
827-859) checked against what the scheme must conserve.

* the hydro variables are bit-identical with and without species (species
  are passive);
* with periodic boundaries the total of every mass scalar (rho * S) is
  conserved to round-off, and so is each species' total;
* the species sum to 1 after every step;
* a uniform scalar stays uniform in a non-uniform flow (the update is
  consistent with the density update), 2D and 3D with the full CTU.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, NUNK
from oracle import orc


def _run(grid, unk, params, steps):
    o = orc.Oracle(params, grid)
    u = unk.copy()
    o.eos_init(u)
    for _ in range(steps):
        st, dt, _ = o.compute_dt(u)
        assert st == 0
        assert o.hydro(u, 0.0, dt, dt) == 0
    return u


@pytest.mark.parametrize("ndim", [2, 3])
def test_species_are_passive_and_conserved(ndim):
    nb, nblk = ((8, 8), (3, 3)) if ndim == 2 else ((8, 8, 8), (2, 2, 2))
    plain = UniformGrid(ndim, nb, nblk, bc="periodic")
    grid = UniformGrid(ndim, nb, nblk, bc="periodic", nspecies=2, nmass_scalars=1)
    params = abi.default_params(gamma=5.0 / 3.0)
    u0 = setups.kelvin_helmholtz(plain)
    u1 = grid.new_unk()
    u1[..., :NUNK] = u0
    setups.add_species(grid, u1)
    a = _run(plain, u0, params, 3)
    b = _run(grid, u1, params, 3)
    assert np.array_equal(grid.interior(a), grid.interior(b)[..., :NUNK])
    it0, it1 = grid.interior(u1), grid.interior(b)
    rho0, rho1 = it0[..., 0], it1[..., 0]
    sp = grid.species
    tot0 = (rho0[..., None] * it0[..., sp]).sum(axis=(0, 1, 2, 3))
    tot1 = (rho1[..., None] * it1[..., sp]).sum(axis=(0, 1, 2, 3))
    np.testing.assert_allclose(tot1, tot0, rtol=1e-12)
    ssum = it1[..., sp.start] + it1[..., sp.start + 1]
    assert np.abs(ssum - 1.0).max() < 1e-14
    assert np.all(it1[..., sp] > -1e-12) and np.all(it1[..., sp.start:sp.start + 2] < 1 + 1e-12)


def test_uniform_scalar_stays_uniform_3d_ctu():
    grid = UniformGrid(3, (8, 8, 8), (2, 2, 2), bc="periodic", nmass_scalars=1)
    params = abi.default_params(gamma=5.0 / 3.0)
    u = grid.new_unk()
    u[..., :NUNK] = setups.kelvin_helmholtz(UniformGrid(3, (8, 8, 8), (2, 2, 2), bc="periodic"))
    grid.interior(u)[..., grid.species.start] = 0.3
    out = _run(grid, u, params, 3)
    s = grid.interior(out)[..., grid.species.start]
    assert np.abs(s - 0.3).max() < 1e-13


def test_species_conserved_on_amr_hierarchy():
    """With the flux correction carrying the species fluxes, the mass
    scalar's total over the leaves (cell volumes of their levels) is
    conserved to round-off on a periodic AMR hierarchy."""
    from flash5_b200.amr import AmrGrid, indicator_refiner
    g = AmrGrid(2, (8, 8), (4, 4), 3, bc="periodic", nspecies=2, nmass_scalars=1)
    f = lambda X, Y, Z: 1.0 + 0.8 * np.tanh(((X - 0.5) ** 2 + (Y - 0.45) ** 2 - 0.04) / 0.004)
    g.refine_levels(indicator_refiner(g, f, 0.05))
    assert g.max_used_level == 3
    params = abi.default_params(gamma=5.0 / 3.0)
    u = setups.add_species(g, setups.kelvin_helmholtz(g))
    o = orc.Oracle(params, g)
    o.eos_init(u)
    leaves = g.leaf_ids
    vol = g.cell_volumes()[leaves]
    def total(uu):
        it = g.interior(uu)[leaves]
        return (vol[:, None, None, None, None] * it[..., 0:1] * it[..., g.species]).sum(axis=(0, 1, 2, 3))
    t0 = total(u)
    for _ in range(3):
        st, dt, _ = o.compute_dt(u)
        assert o.hydro(u, 0.0, dt, dt) == 0
    t1 = total(u)
    np.testing.assert_allclose(t1[2], t0[2], rtol=1e-12)
    it = g.interior(u)[leaves]
    assert np.abs(it[..., g.species.start] + it[..., g.species.start + 1] - 1.0).max() < 1e-14
