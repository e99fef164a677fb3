"""The oracle's hydro step on a rank's share of a sharded uniform grid
(test infrastructure only): the same ShardPlan as the GPU driver, ghost
blocks exchanged as numpy arrays through torch.distributed (gloo on CPU),
the oracle advancing the owned blocks only, dt reduced with MIN."""
import numpy as np

from flash5_b200.hydro import next_dt
from flash5_b200.shard import ShardPlan
from oracle import orc


class ShardedOracle:
    def __init__(self, params, grid, dist):
        self.dist = dist
        self.rank, self.nranks = dist.get_rank(), dist.get_world_size()
        self.plan = ShardPlan(grid, self.nranks, self.rank)
        self.lgrid = self.plan.local_grid()
        self.o = orc.Oracle(params, self.lgrid)
        self.o_owned = orc.Oracle(params, self.plan.owned_grid())
        self.owned = self.plan.owned_local()

    def scatter(self, unk_global):
        """This rank's local UNK (owned + ghosts) from a global UNK."""
        return np.ascontiguousarray(unk_global[self.plan.local])

    def exchange(self, unk):
        """Refresh the ghost blocks' interiors from their owners."""
        import torch
        it = self.lgrid.interior(unk)
        ops, rbufs = [], {}
        for r in sorted(self.plan.send):
            idx = [self.plan.local_of[g] for g in self.plan.send[r]]
            if idx:
                ops.append(self.dist.P2POp(self.dist.isend, torch.from_numpy(np.ascontiguousarray(it[idx])), r))
        for r in sorted(self.plan.recv):
            idx = [self.plan.local_of[g] for g in self.plan.recv[r]]
            if idx:
                rbufs[r] = (idx, torch.empty((len(idx),) + it.shape[1:], dtype=torch.float64))
                ops.append(self.dist.P2POp(self.dist.irecv, rbufs[r][1], r))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        for r, (idx, buf) in rbufs.items():
            it[idx] = buf.numpy()

    def compute_dt(self, unk):
        import torch
        st, dt, loc = self.o_owned.compute_dt(np.ascontiguousarray(unk[self.owned]))
        t = torch.tensor([dt], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())

    def step(self, unk, t, dt, dt_old):
        self.exchange(unk)
        return self.o.hydro(unk, t, dt, dt_old, blocks=self.owned)

    def gather(self, unk, root=0):
        """Owned blocks of every rank assembled into the global order on root."""
        import torch
        mine = torch.from_numpy(np.ascontiguousarray(unk[self.owned]))
        if self.rank != root:
            self.dist.send(mine, root)
            return None
        n = self.plan.grid.nblocks
        out = np.zeros((n,) + unk.shape[1:])
        for r in range(self.nranks):
            ids = self.plan.owned_of(r)
            if r == root:
                out[ids] = mine.numpy()
            else:
                buf = torch.empty((len(ids),) + unk.shape[1:], dtype=torch.float64)
                self.dist.recv(buf, r)
                out[ids] = buf.numpy()
        return out
