"""The product's sharded step across processes (marked gpu).

Two (or three) ranks run as separate processes over a gloo process group on
one GPU; each holds a ShardedHydro context on its share of the grid.  The
ghost blocks travel through the product's own path -- the pack kernel,
pinned host copies, gloo point-to-point messages, the unpack kernel -- and,
with `overlap`, the step runs in two phases around the messages
(flash_hy_step_phase: owned blocks that read no ghost block first, the rest
after the unpack).  No kernel waits on another rank: every exchange passes
through the host.  Each rank also steps the whole grid in one context and
requires its owned blocks to match it bit for bit and the time steps to be
equal; the MINLOC location names a block owned by the rank it reports as
meshMe.
"""
import os
import socket

import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def kh3d():
    g = UniformGrid(3, (8, 8, 8), (4, 3, 3), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0)


def sod3d_mixed():
    g = UniformGrid(3, (8, 8, 8), (3, 3, 2), bc=["outflow", "outflow", "reflecting", "reflecting", "periodic",
                                                  "periodic"])
    return g, setups.sod(g, xangle=30.0, yangle=70.0), abi.default_params(precision=abi.PREC_MIXED)


def _worker(rank, world, port, case, overlap, nsteps, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        from flash5_b200.hydro import Hydro, next_dt
        from flash5_b200.shard import ShardedHydro
        grid, unk, params = case()
        single = Hydro(params, grid)
        single.upload(unk)
        sh = ShardedHydro(params, grid, world, rank, device=0, dist=dist, overlap=overlap)
        sh.upload(unk)
        dt1, loc1 = single.compute_dt()
        dts, locs = sh.compute_dt()
        # equal time steps; the location is a block the reporting rank owns
        # (with ties the ranks' choice may differ from the single context's)
        ok = [dt1 == dts, sh.plan.owner[locs[5]] == locs[4]]
        t, dt_old, dt = 0.0, dt1, dt1
        for _ in range(nsteps):
            single(t + dt, dt, dt_old)
            sh(t + dt, dt, dt_old)
            t += dt
            d1, l1 = single.compute_dt()
            ds, ls = sh.compute_dt()
            ok += [d1 == ds, sh.plan.owner[ls[5]] == ls[4]]
            dt_old, dt = dt, next_dt(d1, dt)
        out = grid.new_unk()
        single.download(out)
        part, ids = sh.download_owned()
        same = bool(np.array_equal(grid.interior(part), grid.interior(out)[ids]))
        launches = sh.last_launch_count
        sh.close()
        single.close()
        q.put((rank, all(ok) and same, ok, same, launches))
    except Exception as e:           # report to the parent instead of hanging it
        q.put((rank, False, repr(e), False, 0))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("case,world,overlap", [(kh3d, 2, True), (kh3d, 3, True), (kh3d, 2, False),
                                                (sod3d_mixed, 2, True)])
def test_sharded_hydro_across_processes(case, world, overlap):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, overlap, 3, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, passed, ok, same, _ in sorted(results, key=lambda r: r[0]):
        assert passed, (rank, ok, same)
