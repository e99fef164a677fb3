"""UNK upload / download through the C ABI (marked gpu).

flash_hy_upload moves only the variables the device needs and
flash_hy_download writes back only the variables the device owns: the
caller's guard cells and the variables it does not own (SHOK) keep their
values, in both of FLASH's UNK layouts (unk(var,i,j,k,blk) and the
--index-reorder unk(i,j,k,var,blk)), with the host-side gather / scatter
split over several threads on larger grids.  The owned variables must equal
the oracle's EOS-consistent UNK (Grid_initDomain's EOS, Eos_putData) bit for
bit.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro
from oracle import orc

OWNED = ("dens", "velx", "vely", "velz", "eint", "ener", "pres", "temp", "gamc", "game")


def _expected_interior(make_grid, fill, params):
    """The oracle's EOS-consistent interiors (the oracle works on FLASH's
    guard-inclusive UNK, so on a twin grid with NGUARD = 4)."""
    g4 = make_grid(4)
    ref = fill(g4)
    orc.Oracle(abi.with_species(params, g4), g4).eos_init(ref)
    return g4.interior(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nguard", [4, 0])
@pytest.mark.parametrize("layout", [abi.LAYOUT_VAR_FASTEST, abi.LAYOUT_XYZ_FASTEST])
def test_round_trip_keeps_guard_cells_and_unowned_variables(nguard, layout):
    def make_grid(ng):
        return UniformGrid(3, (8, 8, 8), (3, 2, 2), bc="periodic", nguard=ng, nspecies=2, nmass_scalars=1)

    def fill(g):
        return setups.add_species(g, setups.kelvin_helmholtz(g))
    grid = make_grid(nguard)
    params = abi.default_params(gamma=5.0 / 3.0)
    unk = fill(grid)
    iw = _expected_interior(make_grid, fill, params)
    h = Hydro(params, grid)
    try:
        host = np.ascontiguousarray(np.moveaxis(unk, -1, 1)) if layout == abi.LAYOUT_XYZ_FASTEST else unk
        h.upload(host, layout=layout)
        out = np.full_like(host, -7.25)             # sentinel in guard cells and SHOK
        h.download(out, layout=layout)
    finally:
        h.close()
    if layout == abi.LAYOUT_XYZ_FASTEST:
        out = np.ascontiguousarray(np.moveaxis(out, 1, -1))
    it = grid.interior(out)
    for v in OWNED:
        assert np.array_equal(it[..., VAR[v]], iw[..., VAR[v]]), v
    for q in range(3):
        k = grid.species.start + q
        assert np.array_equal(it[..., k], iw[..., k]), ("species", q)
    assert np.all(it[..., VAR["shok"]] == -7.25)
    if nguard:
        mask = np.ones(out.shape[:4], dtype=bool)
        g = grid.ng
        mask[:, g[2]:g[2] + grid.nb[2], g[1]:g[1] + grid.nb[1], g[0]:g[0] + grid.nb[0]] = False
        assert np.all(out[mask] == -7.25)


@pytest.mark.gpu
def test_threaded_transfers_on_a_larger_grid():
    # 4096 blocks: the gather / scatter runs on several host threads, each
    # with its own stream and pinned sub-chunk slots
    def make_grid(ng):
        return UniformGrid(3, (8, 8, 8), (16, 16, 16), bc="periodic", nguard=ng)
    grid = make_grid(0)
    params = abi.default_params(gamma=5.0 / 3.0)
    unk = setups.kelvin_helmholtz(grid)
    want = _expected_interior(make_grid, setups.kelvin_helmholtz, params)
    h = Hydro(params, grid)
    try:
        for _ in range(2):                          # the second call reuses the pool
            h.upload(unk)
            out = np.zeros_like(unk)
            h.download(out)
            for v in OWNED:
                assert np.array_equal(grid.interior(out)[..., VAR[v]], want[..., VAR[v]]), v
    finally:
        h.close()
