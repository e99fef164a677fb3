"""The FLASH-facing conventions of the C ABI, called directly through ctypes
(marked gpu).

* Block lists and block IDs are FLASH's 1-based IDs (blockList(1:blockCount)
  of Hydro(blockCount, blockList, ...), Grid_getFluxData(blockID, ...)):
  flash_hy_step_blocks with IDs b + 1 advances exactly the oracle's blocks b,
  bit for bit; IDs 0 and nblocks + 1 are refused.
* The dt location is FLASH's dtMinLoc (i, j, k, level, meshMe)
  (Hydro_computeDt.F90:266-270): meshMe is 0 until flash_hy_set_mesh_me
  sets it; flash_hy_dt_block gives the 1-based ID of the limiting block.
"""
import ctypes as C

import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.grid import VAR
from flash5_b200.hydro import Hydro
from oracle import orc
from tests.cases import make_case


@pytest.mark.gpu
def test_block_ids_are_one_based_through_the_c_abi():
    grid, unk, params = make_case("sod2d_rot")
    lib = abi.load_library()
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    try:
        h.upload(unk)
        st, dt, loc = o.compute_dt(ref)
        blocks = [1, 5, 6, 10, grid.nblocks - 1]
        ids = (C.c_int * len(blocks))(*[b + 1 for b in blocks])
        assert lib.flash_hy_step_blocks(h.ctx, len(blocks), ids, dt, dt, dt, 0) == 0
        assert o.hydro(ref, dt, dt, dt, blocks=blocks) == 0
        out = grid.new_unk()
        h.download(out)
        for v in ("dens", "velx", "vely", "eint", "ener", "pres"):
            assert np.array_equal(grid.interior(out)[..., VAR[v]], grid.interior(ref)[..., VAR[v]]), v
        for bad in (0, grid.nblocks + 1, -3):
            one = (C.c_int * 1)(bad)
            assert lib.flash_hy_step_blocks(h.ctx, 1, one, dt, dt, dt, 0) == abi.ERR_BAD_ARG
            assert lib.flash_hy_compute_fluxes(h.ctx, 1, one, dt, abi.UPDATE_NONE) == abi.ERR_BAD_ARG
        one = (C.c_int * 1)(3)
        assert lib.flash_hy_compute_fluxes(h.ctx, 1, one, dt, abi.UPDATE_NONE) == 0
        nb = grid.nb
        flx = np.zeros(((nb[0] + 1) * nb[1] * nb[2], 8))
        fp = flx.ctypes.data_as(C.POINTER(C.c_double))
        assert lib.flash_hy_get_fluxes(h.ctx, 3, 1, fp) == 0
        st, want = o.block_fluxes(ref.copy(), 2, dt)
        assert st == 0 and np.array_equal(flx, want[0])
        assert lib.flash_hy_get_fluxes(h.ctx, 0, 1, fp) == abi.ERR_BAD_ARG
        assert lib.flash_hy_put_fluxes(h.ctx, grid.nblocks + 1, 1, fp) == abi.ERR_BAD_ARG
    finally:
        h.close()


@pytest.mark.gpu
def test_dt_location_carries_mesh_rank_and_block_id():
    grid, unk, params = make_case("kh3d")
    lib = abi.load_library()
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    _, dto, loco = o.compute_dt(ref)
    h = Hydro(params, grid)
    try:
        h.upload(unk)
        dt, loc, bid = C.c_double(), (C.c_int * 5)(), C.c_int()
        assert lib.flash_hy_compute_dt(h.ctx, C.byref(dt), loc) == 0
        assert dt.value == dto and tuple(loc) == tuple(loco[:4]) + (0,)
        assert lib.flash_hy_dt_block(h.ctx, C.byref(bid)) == 0 and bid.value == loco[5] + 1
        assert lib.flash_hy_set_mesh_me(h.ctx, 3) == 0
        assert lib.flash_hy_compute_dt(h.ctx, C.byref(dt), loc) == 0
        assert tuple(loc) == tuple(loco[:4]) + (3,)
        assert lib.flash_hy_set_mesh_me(h.ctx, -1) == abi.ERR_BAD_ARG
    finally:
        h.close()
