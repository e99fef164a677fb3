"""flash_hy_compute_dt_noalloc: the CFL time step for callers that cannot
allocate device memory (marked gpu).

Such callers own the device state themselves (inside another framework's
memory pool, or under an allocation budget fixed at start-up), so the entry
point takes their device arrays and uses only its fixed file-scope scratch.
Checked here through the C ABI against the context-based flash_hy_compute_dt,
bit for bit, on two consecutive calls (two different states): on small grids
in 2D and 3D, and on the 2D Sod grid of 32 x 32 blocks, whose 1024 blocks
take the reduction's strided loop and, with its many equal time steps, the
tie-break across threads.  Also: the call allocates no device memory (free
memory unchanged over repeated calls), it runs on a caller's non-default
stream, and grids larger than the fixed scratch are refused.  Collected last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro


def _noalloc_fn():
    lib = abi.load_library()
    f = lib.flash_hy_compute_dt_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 5 + [C.c_int] * 5 + [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_void_p,
                                                     C.POINTER(C.c_double), C.POINTER(C.c_int)]
    return f


def _call(f, arrays, grid, gamma, cfl, nblocks=None, stream=None):
    dt = C.c_double()
    loc = (C.c_int * 5)()
    deltas = (C.c_double * 3)(*grid.delta)
    st = f(*[a.data_ptr() for a in arrays], grid.ndim, grid.nb[0], grid.nb[1], grid.nb[2],
           grid.nblocks if nblocks is None else nblocks, deltas, gamma, cfl, stream, C.byref(dt), loc)
    return st, dt.value, tuple(loc)


def _device_state(h, grid):
    import torch
    out = grid.new_unk()
    h.download(out)
    it = grid.interior(out)
    return [torch.tensor(np.ascontiguousarray(it[..., VAR[v]]), dtype=torch.float64, device="cuda:0")
            for v in ("dens", "velx", "vely", "velz", "eint")]


def _case(name):
    if name == "kh3d":
        grid = UniformGrid(3, (8, 8, 8), (3, 2, 2), bc="periodic", nguard=0)
        return grid, setups.kelvin_helmholtz(grid, gamma=5.0 / 3.0), 5.0 / 3.0
    if name == "kh2d_16":
        grid = UniformGrid(2, (16, 16), (3, 2), bc="periodic", nguard=0)
        return grid, setups.kelvin_helmholtz(grid, gamma=5.0 / 3.0), 5.0 / 3.0
    grid = UniformGrid(2, (8, 8), (32, 32), bc="outflow", nguard=0)     # 2D Sod, 256^2 as 32 x 32 blocks
    return grid, setups.sod(grid), 1.4


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["kh3d", "kh2d_16", "sod2d_1024"])
def test_noalloc_dt_matches_context_dt(name):
    import torch
    torch.cuda.set_device(0)
    grid, unk, gamma = _case(name)
    params = abi.default_params(gamma=gamma)
    h = Hydro(params, grid)
    h.upload(unk)
    f = _noalloc_fn()
    t, dt_old = 0.0, None
    try:
        for call in range(2):
            dt_ctx, loc_ctx = h.compute_dt()
            arrays = _device_state(h, grid)
            st, dt, loc = _call(f, arrays, grid, gamma, params.cfl)
            assert st == 0
            assert dt == dt_ctx, (call, dt, dt_ctx)
            # the context reports (i, j, k, level, meshMe) and the block
            # separately; this entry point reports (i, j, k, level, block)
            assert loc == tuple(loc_ctx[:4]) + (loc_ctx[5],), (call, loc, loc_ctx)
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


@pytest.mark.gpu
def test_noalloc_allocates_nothing_and_runs_on_caller_stream():
    import torch
    torch.cuda.set_device(0)
    grid, unk, gamma = _case("sod2d_1024")
    params = abi.default_params(gamma=gamma)
    h = Hydro(params, grid)
    h.upload(unk)
    try:
        dt_ctx, loc_ctx = h.compute_dt()
        arrays = _device_state(h, grid)
    finally:
        h.close()
    f = _noalloc_fn()
    want = (0, dt_ctx, tuple(loc_ctx[:4]) + (loc_ctx[5],))
    assert _call(f, arrays, grid, gamma, params.cfl) == want          # warm: first call in this context
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(5):
        assert _call(f, arrays, grid, gamma, params.cfl) == want
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        got = _call(f, arrays, grid, gamma, params.cfl, stream=s.cuda_stream)
    assert got == want


def abi_max_blocks():
    import os
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "flash_hy.h")).read()
    for line in hdr.splitlines():
        if line.startswith("#define FLASH_HY_NOALLOC_MAX_BLOCKS"):
            return int(line.split()[2])
    raise AssertionError("FLASH_HY_NOALLOC_MAX_BLOCKS not declared")
