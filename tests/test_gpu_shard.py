"""Sharded grids on one GPU (marked gpu): two or three rank contexts of the
same grid in one process, their ghost blocks moved by device copies between
the ranks' pack and unpack buffers (the exchange NCCL does between GPUs).
The FP64 result must equal the single-context GPU run, and the oracle, bit
for bit -- which exercises partial grids, owned-block stepping, the packing
kernels and the per-rank dt reduction through the C ABI.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid
from flash5_b200.hydro import Hydro, next_dt
from flash5_b200.shard import ShardedHydro
from oracle import orc


def kh3d():
    g = UniformGrid(3, (8, 8, 8), (3, 3, 2), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0)


def kh2d():
    g = UniformGrid(2, (8, 8), (8, 6), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0)


def kh3d_species():
    g = UniformGrid(3, (8, 8, 8), (3, 3, 2), bc="periodic", nspecies=2, nmass_scalars=1)
    return g, setups.add_species(g, setups.kelvin_helmholtz(g)), abi.default_params(gamma=5.0 / 3.0)


def sod2d():
    g = UniformGrid(2, (8, 8), (5, 3), bc=["outflow", "outflow", "reflecting", "reflecting"])
    return g, setups.sod(g, xangle=30.0), abi.default_params()


def exchange_in_process(ranks):
    import torch
    for s in ranks:
        s.pack()
        s.h.sync()
    for s in ranks:
        for r, v in s.send_views.items():
            ranks[r].recv_views[s.rank].copy_(v)
    torch.cuda.synchronize()
    for s in ranks:
        s.unpack()


@pytest.mark.gpu
@pytest.mark.parametrize("case,nranks,prec", [(kh3d, 2, abi.PREC_FP64), (kh3d, 3, abi.PREC_MIXED),
                                              (kh2d, 3, abi.PREC_FP64), (sod2d, 3, abi.PREC_FP64),
                                              (kh3d_species, 3, abi.PREC_FP64)])
def test_sharded_contexts_match_single_context(case, nranks, prec):
    grid, unk, params = case()
    params.precision = prec
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    single = Hydro(params, grid)
    single.upload(unk)
    ranks = [ShardedHydro(params, grid, nranks, r) for r in range(nranks)]
    for s in ranks:
        s.upload(unk)
    dt, loc1 = single.compute_dt()
    got = [s.compute_dt() for s in ranks]
    assert min(g[0] for g in got) == dt
    # each rank reports its own meshMe and the global id of its limiting block
    for r, (dtr, locr) in enumerate(got):
        assert locr[4] == r and ranks[r].plan.owner[locr[5]] == r
    best = min(range(nranks), key=lambda r: (got[r][0], r))
    if sum(g[0] == dt for g in got) == 1:
        assert got[best][1][:4] == loc1[:4] and got[best][1][5] == loc1[5]
    t, dt_old = 0.0, dt
    for _ in range(3):
        single(t + dt, dt, dt_old)
        exchange_in_process(ranks)
        for s in ranks:
            s.h(t + dt, dt, dt_old)
        if prec == abi.PREC_FP64:
            assert o.hydro(ref, t + dt, dt, dt_old) == 0
        t += dt
        dts, _ = single.compute_dt()
        dtr = min(s.compute_dt()[0] for s in ranks)
        assert dtr == dts
        dt_old, dt = dt, next_dt(dts, dt)
    out = grid.new_unk()
    single.download(out)
    got = np.zeros_like(out)
    for s in ranks:
        part, ids = s.download_owned()
        got[ids] = part
        s.close()
    single.close()
    assert np.array_equal(grid.interior(got), grid.interior(out))
    if prec == abi.PREC_FP64:
        assert np.array_equal(grid.interior(got), grid.interior(ref))


@pytest.mark.gpu
def test_partial_grid_needs_owned_blocks():
    from flash5_b200.hydro import HydroError
    from flash5_b200.shard import ShardPlan
    grid = UniformGrid(2, (8, 8), (8, 8), bc="outflow")
    unk, params = setups.sod(grid, xangle=30.0), abi.default_params()
    plan = ShardPlan(grid, 2, 0)
    assert len(plan.local) < grid.nblocks
    h = Hydro(params, plan.local_grid())
    h.upload(np.ascontiguousarray(unk[plan.local]))
    with pytest.raises(HydroError):
        h(1e-4, 1e-4, 1e-4)                        # no owned blocks named yet
    with pytest.raises(HydroError):
        h.set_owned_blocks(np.arange(len(plan.local)))   # ghosts' neighbours are absent
    h.set_owned_blocks(plan.owned_local())
    h(1e-4, 1e-4, 1e-4)
    h.sync()
    h.close()
