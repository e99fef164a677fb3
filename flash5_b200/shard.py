"""Block sharding of a uniform grid across ranks with a ghost-block exchange.

FLASH distributes leaf blocks over MPI ranks along the Morton curve
(PARAMESH `amr_morton_order`, UG process grid) and fills guard cells from
other ranks' blocks once per step (`Grid_fillGuardCells`, `gr_shiftData`);
the time step is a MINLOC all-reduce (`Driver_computeDt.F90:376-377`).  Here
each rank owns a contiguous range of the Morton order and keeps, besides its
own blocks, *ghost blocks*: copies of the other ranks' blocks that touch one
of its blocks (faces, edges, corners; NGUARD = 4 never reaches further than
one block).  One step is: exchange the ghost blocks' interiors, advance the
owned blocks only, reduce dt.

`ShardPlan` is pure host logic (tested with gloo ranks on CPU); the GPU
driver (`ShardedHydro`) moves ghost blocks with the C ABI's pack/unpack
kernels and NCCL point-to-point sends; the oracle driver
(`ShardedOracle`, test infrastructure) moves them as numpy arrays.
"""
import itertools

import numpy as np

from .grid import UniformGrid


def morton_key(c):
    k = 0
    for bit in range(16):
        for d in range(3):
            k |= ((int(c[d]) >> bit) & 1) << (3 * bit + d)
    return k


class LocalGrid(UniformGrid):
    """A rank's share of a uniform grid: owned blocks first, then ghosts,
    with global block coordinates and the global block extents."""

    def __init__(self, ndim, nb, nblk, coords, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), bc="outflow", nguard=4,
                 nspecies=0, nmass_scalars=0):
        super().__init__(ndim, nb, nblk, lo=lo, hi=hi, bc=bc, nguard=nguard, nspecies=nspecies,
                         nmass_scalars=nmass_scalars)
        self.coords = np.ascontiguousarray(np.asarray(coords, dtype=np.int32).reshape(-1, 3))
        self.nblocks = len(self.coords)
        self.levels = np.ones(self.nblocks, dtype=np.int32)


class ShardPlan:
    """Partition of a uniform grid's blocks over `nranks` ranks and the
    ghost exchange of rank `rank`.

    order         global ids in Morton order
    owner[g]      rank owning global block g (g = index in grid.coords)
    owned         global ids owned by this rank, Morton order
    ghosts        global ids this rank needs from others, grouped by owner
    recv[r]       global ids received from rank r (in local ghost order)
    send[r]       global ids of this rank's blocks that rank r needs, in the
                  order rank r lists them in its recv[this rank]
    local_of[g]   local index of a global block (owned, then ghosts)
    """

    def __init__(self, grid, nranks, rank):
        self.grid, self.nranks, self.rank = grid, nranks, rank
        n = grid.nblocks
        order = sorted(range(n), key=lambda g: morton_key(grid.coords[g]))
        self.order = order
        self.owner = np.empty(n, dtype=np.int32)
        bounds = [round(i * n / nranks) for i in range(nranks + 1)]
        for r in range(nranks):
            for g in order[bounds[r]:bounds[r + 1]]:
                self.owner[g] = r
        self._at = {tuple(int(v) for v in grid.coords[g]): g for g in range(n)}
        self.owned = [g for g in order if self.owner[g] == rank]
        # adjacency is symmetric, so this rank's neighbour lists give both
        # what it receives (touching blocks of other ranks) and what it sends
        # (its blocks touching another rank's block)
        recv = {r: set() for r in range(nranks) if r != rank}
        send = {r: set() for r in range(nranks) if r != rank}
        for g in self.owned:
            for h in self.neighbors(g):
                r = int(self.owner[h])
                if r != rank:
                    recv[r].add(h)
                    send[r].add(g)
        self.recv = {r: sorted(v) for r, v in recv.items()}
        self.send = {r: sorted(v) for r, v in send.items()}
        self.ghosts = [g for r in sorted(self.recv) for g in self.recv[r]]
        self.local = self.owned + self.ghosts
        self.local_of = {g: i for i, g in enumerate(self.local)}

    def neighbors(self, g):
        """Global ids of the blocks touching block g (boundary conditions
        applied: periodic wraps, other boundaries have no neighbour)."""
        grid = self.grid
        c = grid.coords[g]
        out = set()
        for o in itertools.product((-1, 0, 1), repeat=grid.ndim):
            if not any(o):
                continue
            p = [int(c[d]) for d in range(3)]
            ok = True
            for d in range(grid.ndim):
                p[d] += o[d]
                if p[d] < 0 or p[d] >= grid.nblk[d]:
                    if grid.bc[2 * d] == -135:
                        p[d] %= grid.nblk[d]
                    else:
                        ok = False
            if ok:
                out.add(self._at[tuple(p)])
        out.discard(g)
        return out

    def local_grid(self):
        gr = self.grid
        return LocalGrid(gr.ndim, gr.nb[:gr.ndim], gr.nblk[:gr.ndim], gr.coords[self.local], lo=gr.lo, hi=gr.hi,
                         bc=gr.bc, nguard=gr.nguard, nspecies=gr.nspecies, nmass_scalars=gr.nmass_scalars)

    def owned_of(self, r):
        """Global ids owned by rank r, in its local (Morton) order."""
        return [g for g in self.order if self.owner[g] == r]

    def owned_grid(self):
        """The owned blocks alone (for reductions over owned blocks)."""
        gr = self.grid
        return LocalGrid(gr.ndim, gr.nb[:gr.ndim], gr.nblk[:gr.ndim], gr.coords[self.owned], lo=gr.lo, hi=gr.hi,
                         bc=gr.bc, nguard=gr.nguard, nspecies=gr.nspecies, nmass_scalars=gr.nmass_scalars)

    def owned_local(self):
        return np.arange(len(self.owned), dtype=np.int32)

    def send_local(self):
        """Local indices of the blocks sent, rank by rank (ascending rank)."""
        return np.array([self.local_of[g] for r in sorted(self.send) for g in self.send[r]], dtype=np.int32)

    def recv_local(self):
        """Local indices of the ghost blocks received, rank by rank."""
        return np.array([self.local_of[g] for r in sorted(self.recv) for g in self.recv[r]], dtype=np.int32)


class ShardedHydro:
    """One rank's GPU context on its share of a sharded grid.

    The ghost blocks travel as device buffers: `pack` gathers the blocks
    other ranks need (one kernel on the context's stream), the buffers move
    rank to rank (NCCL point-to-point sends through torch.distributed, or
    pinned host copies over a gloo group, or any other transport through
    `send_views` / `recv_views`), `unpack` scatters the received blocks into
    the ghost slots.  With a process group the step overlaps the exchange
    (`overlap`, the default): the owned blocks that read no ghost block
    advance while the messages are in flight (flash_hy_step_phase 1), the
    others after the unpack (phase 2).  `compute_dt` reduces dt over the
    owned blocks and, with a process group, does Driver_computeDt's
    MPI_MINLOC over the ranks."""

    def __init__(self, params, grid, nranks, rank, device=0, dist=None, overlap=True):
        import torch
        from .hydro import Hydro
        self.torch, self.dist, self.device = torch, dist, device
        self.nranks, self.rank = nranks, rank
        self.plan = ShardPlan(grid, nranks, rank)
        self.lgrid = self.plan.local_grid()
        self.h = Hydro(params, self.lgrid, device=device)
        self.h.set_mesh_me(rank)
        self.h.set_owned_blocks(self.plan.owned_local())
        send, recv = self.plan.send_local(), self.plan.recv_local()
        self.h.set_exchange(send, recv)
        per = (5 + grid.nspecies + grid.nmass_scalars) * grid.nb[0] * grid.nb[1] * grid.nb[2]
        dev = torch.device("cuda", device)
        self.sbuf = torch.empty(max(1, len(send)) * per, dtype=torch.float64, device=dev)
        self.rbuf = torch.empty(max(1, len(recv)) * per, dtype=torch.float64, device=dev)
        self.send_views, self.recv_views = {}, {}
        off = 0
        for r in sorted(self.plan.send):
            k = len(self.plan.send[r])
            if k:
                self.send_views[r] = self.sbuf[off * per:(off + k) * per]
            off += k
        off = 0
        for r in sorted(self.plan.recv):
            k = len(self.plan.recv[r])
            if k:
                self.recv_views[r] = self.rbuf[off * per:(off + k) * per]
            off += k
        self._tstream = torch.cuda.ExternalStream(self.h.stream, device=dev)
        self.overlap = overlap
        # gloo carries CPU tensors: the ghost buffers go through pinned host copies
        self.host_transport = dist is not None and dist.get_backend() == "gloo"
        self.coll_device = torch.device("cpu") if self.host_transport else dev
        if self.host_transport:
            self.sbuf_h = torch.empty(self.sbuf.numel(), dtype=torch.float64, pin_memory=True)
            self.rbuf_h = torch.empty(self.rbuf.numel(), dtype=torch.float64, pin_memory=True)
            self.send_views_h = {r: self.sbuf_h[v.storage_offset():v.storage_offset() + v.numel()]
                                 for r, v in self.send_views.items()}
            self.recv_views_h = {r: self.rbuf_h[v.storage_offset():v.storage_offset() + v.numel()]
                                 for r, v in self.recv_views.items()}

    def upload(self, unk_global):
        """Upload this rank's blocks (owned + ghosts) taken from a global UNK
        (or an already local one when its length matches)."""
        unk = unk_global if len(unk_global) == self.lgrid.nblocks and len(unk_global) != len(self.plan.owner) \
            else unk_global[self.plan.local]
        self.h.upload(np.ascontiguousarray(unk))

    def pack(self):
        self.h.pack(self.sbuf)

    def unpack(self):
        self.h.unpack(self.rbuf)

    def post_exchange(self):
        """Pack the blocks other ranks need and post the point-to-point
        messages; returns the pending requests (finish_exchange completes
        them).  NCCL: device buffers, the messages run on NCCL's stream after
        the pack.  gloo: the packed buffer is copied to pinned host memory
        first."""
        torch, dist = self.torch, self.dist
        self.pack()
        cur = torch.cuda.current_stream(self.device)
        cur.wait_stream(self._tstream)
        if self.host_transport:
            # the copies run on torch's own stream: the pinned buffers' cached
            # blocks must never refer to the context's stream, which dies with it
            self.sbuf_h.copy_(self.sbuf, non_blocking=True)
            cur.synchronize()
            sv, rv = self.send_views_h, self.recv_views_h
        else:
            sv, rv = self.send_views, self.recv_views
        ops = [dist.P2POp(dist.isend, v, r) for r, v in sv.items()]
        ops += [dist.P2POp(dist.irecv, v, r) for r, v in rv.items()]
        return dist.batch_isend_irecv(ops) if ops else []

    def finish_exchange(self, reqs):
        """Complete the messages and unpack the ghost blocks (ordered on the
        context's stream after whatever it already holds)."""
        torch = self.torch
        for w in reqs:
            w.wait()
        cur = torch.cuda.current_stream(self.device)
        if self.host_transport:
            self.rbuf.copy_(self.rbuf_h, non_blocking=True)
        self._tstream.wait_stream(cur)
        self.unpack()

    def exchange(self):
        """Ghost exchange over the process group, blocking."""
        self.finish_exchange(self.post_exchange())

    def __call__(self, simTime, dt, dtOld, sweepOrder=0):
        if self.nranks > 1 and self.dist is not None:
            if self.overlap:
                reqs = self.post_exchange()
                self.h.step_phase(simTime, dt, dtOld, 1)     # blocks that read no ghost block
                self.finish_exchange(reqs)
                self.h.step_phase(simTime, dt, dtOld, 2)
                return
            self.exchange()
        self.h(simTime, dt, dtOld, sweepOrder)

    def compute_dt(self):
        """(dt, (i, j, k, level, meshMe, block)): dt over the owned blocks;
        with a process group, the MPI_MINLOC of Driver_computeDt.F90:376-423
        -- the minimum over ranks, and the location of the lowest rank that
        holds it, broadcast from that rank.  block is the global block id."""
        dt, loc = self.h.compute_dt()
        loc = loc[:5] + (int(self.plan.local[loc[5]]) if loc[5] >= 0 else -1,)
        if self.nranks > 1 and self.dist is not None:
            torch, dist = self.torch, self.dist
            dev = self.coll_device
            t = torch.tensor([dt], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            gdt = float(t.item())
            w = torch.tensor([self.rank if dt == gdt else self.nranks], dtype=torch.int64, device=dev)
            dist.all_reduce(w, op=dist.ReduceOp.MIN)
            lt = torch.tensor(loc, dtype=torch.int64, device=dev)
            dist.broadcast(lt, src=int(w.item()))
            dt, loc = gdt, tuple(int(x) for x in lt.tolist())
        return dt, loc

    @property
    def stream(self):
        return self.h.stream

    @property
    def last_launch_count(self):
        """Launches of the last step, the ghost pack and unpack included
        (an overlapped step launches the step's kernels once per phase)."""
        if self.nranks > 1 and self.dist is not None:
            return self.h.last_launch_count * (2 if self.overlap else 1) + 2
        return self.h.last_launch_count

    def download_owned(self):
        """UNK of the owned blocks (local order = Morton order) and their
        global ids."""
        out = self.lgrid.new_unk()
        self.h.download(out)
        return out[:len(self.plan.owned)], list(self.plan.owned)

    def close(self):
        self.h.close()
