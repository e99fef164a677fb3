"""Block sharding across ranks (CPU, gloo, world size 2 and 3).

The exchange plan (flash5_b200/shard.py) is checked for completeness and
symmetry, and the sharded step -- ghost blocks exchanged with
torch.distributed point-to-point messages, owned blocks advanced by the
oracle, dt reduced with MIN -- must reproduce the single-domain oracle run
bit for bit.
"""
import os
import socket

import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid
from flash5_b200.shard import ShardPlan


def test_plan_covers_every_neighbour_and_is_symmetric():
    g = UniformGrid(3, (8, 8, 8), (4, 3, 3), bc=["periodic", "periodic", "outflow", "outflow", "reflecting",
                                                 "reflecting"])
    nr = 3
    plans = [ShardPlan(g, nr, r) for r in range(nr)]
    owned = [set(p.owned) for p in plans]
    assert set().union(*owned) == set(range(g.nblocks)) and sum(len(o) for o in owned) == g.nblocks
    for r, p in enumerate(plans):
        local = set(p.local)
        for b in p.owned:
            assert p.neighbors(b) <= local
        for q in range(nr):
            if q != r:
                assert p.send[q] == plans[q].recv[r]
    lg = plans[0].local_grid()
    assert lg.nblocks == len(plans[0].local)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, case, nsteps, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.shard_oracle import ShardedOracle
        grid, unk, params = case()
        from oracle import orc
        orc.Oracle(params, grid).eos_init(unk)
        so = ShardedOracle(params, grid, dist)
        loc = so.scatter(unk)
        dt = so.compute_dt(loc)
        t, dt_old, dts = 0.0, dt, []
        for _ in range(nsteps):
            assert so.step(loc, t + dt, dt, dt_old) == 0
            t += dt
            dcfl = so.compute_dt(loc)
            dts.append(dcfl)
            dt_old, dt = dt, min(dcfl, 2 * dt)
        out = so.gather(loc)
        if rank == 0:
            q.put((out, dts))
    finally:
        dist.destroy_process_group()


def kh2d():
    g = UniformGrid(2, (8, 8), (4, 3), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0)


def sod3d():
    g = UniformGrid(3, (8, 8, 8), (3, 2, 2), bc=["outflow", "outflow", "reflecting", "reflecting", "periodic",
                                                  "periodic"])
    return g, setups.sod(g, xangle=30.0, yangle=70.0), abi.default_params()


@pytest.mark.parametrize("case,world", [(kh2d, 2), (kh2d, 3), (sod3d, 2)])
def test_sharded_oracle_matches_single_domain(case, world):
    import torch.multiprocessing as mp
    from oracle import orc
    nsteps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out, dts = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    grid, ref, params = case()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    _, dt, _ = o.compute_dt(ref)
    t, dt_old = 0.0, dt
    for n in range(nsteps):
        assert o.hydro(ref, t + dt, dt, dt_old) == 0
        t += dt
        _, dcfl, _ = o.compute_dt(ref)
        assert dcfl == dts[n]
        dt_old, dt = dt, min(dcfl, 2 * dt)
    assert np.array_equal(grid.interior(out), grid.interior(ref))
