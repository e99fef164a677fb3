"""flash_hy_compute_dt_noalloc: the CFL time step for callers that cannot
allocate device memory (marked gpu).

Such callers own the device state themselves (e.g. inside another
framework's memory pool, under a fixed allocation budget, or while
capturing a stream into a graph), so the entry point takes their device
arrays and uses only its fixed file-scope scratch.  Checked here through the
C ABI against the context-based flash_hy_compute_dt, bit for bit, on two
consecutive calls (two different states), plus the rejection of grids
larger than the fixed scratch.  Collected last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro, next_dt


def _noalloc_fn():
    lib = abi.load_library()
    f = lib.flash_hy_compute_dt_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 5 + [C.c_int] * 5 + [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_void_p,
                                                     C.POINTER(C.c_double), C.POINTER(C.c_int)]
    return f


def _call(f, arrays, grid, gamma, cfl, nblocks=None):
    dt = C.c_double()
    loc = (C.c_int * 5)()
    deltas = (C.c_double * 3)(*grid.delta)
    st = f(*[a.data_ptr() for a in arrays], grid.ndim, grid.nb[0], grid.nb[1], grid.nb[2],
           grid.nblocks if nblocks is None else nblocks, deltas, gamma, cfl, None, C.byref(dt), loc)
    return st, dt.value, tuple(loc)


@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [3, 2])
def test_noalloc_dt_matches_context_dt(ndim):
    import torch
    torch.cuda.set_device(0)
    if ndim == 3:
        grid = UniformGrid(3, (8, 8, 8), (3, 2, 2), bc="periodic", nguard=0)
    else:
        grid = UniformGrid(2, (16, 16), (3, 2), bc="periodic", nguard=0)
    gamma = 5.0 / 3.0
    params = abi.default_params(gamma=gamma)
    h = Hydro(params, grid)
    h.upload(setups.kelvin_helmholtz(grid, gamma=gamma))
    f = _noalloc_fn()
    t, dt_old = 0.0, None
    try:
        for call in range(2):
            dt_ctx, loc_ctx = h.compute_dt()
            out = grid.new_unk()
            h.download(out)
            it = grid.interior(out)
            arrays = [torch.tensor(np.ascontiguousarray(it[..., VAR[v]]), dtype=torch.float64, device="cuda:0")
                      for v in ("dens", "velx", "vely", "velz", "eint")]
            st, dt, loc = _call(f, arrays, grid, gamma, params.cfl)
            assert st == 0
            assert dt == dt_ctx, (call, dt, dt_ctx)
            assert loc == tuple(loc_ctx), (call, loc, loc_ctx)
            # the shared scratch keeps the last call's contents; a repeat
            # call on the same state gives the same answer
            st2, dt2, loc2 = _call(f, arrays, grid, gamma, params.cfl)
            assert (st2, dt2, loc2) == (st, dt, loc)
            dt_old = dt if dt_old is None else dt_old
            h(t + dt, dt, dt_old)
            t += dt
            dt_old = dt
        # grids beyond the fixed scratch are refused before any launch
        st, _, _ = _call(f, arrays, grid, gamma, params.cfl, nblocks=abi_max_blocks() + 1)
        assert st == abi.ERR_BAD_ARG
    finally:
        h.close()


def abi_max_blocks():
    import os
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "flash_hy.h")).read()
    for line in hdr.splitlines():
        if line.startswith("#define FLASH_HY_NOALLOC_MAX_BLOCKS"):
            return int(line.split()[2])
    raise AssertionError("FLASH_HY_NOALLOC_MAX_BLOCKS not declared")
