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
