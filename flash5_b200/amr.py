"""Block-structured AMR hierarchy in PARAMESH form.

Every node of the refinement tree is a block of ``nb`` interior cells, as in
PARAMESH (paramesh4/Paramesh4dev/PM4_package): a parent holds the
restriction of its children, the leaves are the blocks Hydro advances
(Grid_getTileIterator(LEAF), unsplit/Hydro.F90:149-229).  Level 1 is the
complete root grid of ``nblk`` blocks per axis; a block at level l has
block coordinates on the level-l grid of nblk * 2**(l-1) blocks per axis
and cell size delta_1 / 2**(l-1).  Refinement keeps PARAMESH's 2:1 balance
across faces, edges and corners (diagonals = .true., Paramesh4dev/Config:
133-134), so every leaf touches only leaves one level up or down.

Nodes are numbered level by level, Morton order inside a level; the host
UNK array holds every node (shape (nblocks, nzt, nyt, nxt, NUNK)), like
FLASH's unk(:,:,:,:,1:lnblocks) with parents included.
"""
import ctypes as C
import copy
import itertools

import numpy as np

from . import abi
from .grid import NGUARD, NUNK, VAR


def _morton(c):
    k = 0
    for bit in range(16):
        for d in range(3):
            k |= ((c[d] >> bit) & 1) << (3 * bit + d)
    return k


class AmrGrid:
    def __init__(self, ndim, nb, nblk, max_level, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), bc="outflow",
                 nguard=NGUARD, nspecies=0, nmass_scalars=0):
        self.ndim = ndim
        self.nspecies, self.nmass_scalars = int(nspecies), int(nmass_scalars)
        self.nunk = NUNK + self.nspecies + self.nmass_scalars
        nb = tuple(nb) + (1,) * (3 - len(nb))
        nblk = tuple(nblk) + (1,) * (3 - len(nblk))
        self.nb = tuple(nb[d] if d < ndim else 1 for d in range(3))
        self.nblk = tuple(nblk[d] if d < ndim else 1 for d in range(3))
        self.max_level = int(max_level)
        self.lo, self.hi = tuple(lo), tuple(hi)
        if isinstance(bc, str):
            bc = [bc] * 6
        code = {"outflow": abi.BC_OUTFLOW, "periodic": abi.BC_PERIODIC, "reflecting": abi.BC_REFLECTING}
        self.bc = [code[b] if isinstance(b, str) else int(b) for b in bc]
        self.periodic = [self.bc[2 * d] == abi.BC_PERIODIC for d in range(3)]
        self.nguard = nguard
        self.ng = (nguard, nguard if ndim > 1 else 0, nguard if ndim > 2 else 0)
        self.nt = tuple(self.nb[d] + 2 * self.ng[d] for d in range(3))
        self.delta1 = tuple((self.hi[d] - self.lo[d]) / (self.nblk[d] * self.nb[d]) if d < ndim else 1.0
                            for d in range(3))
        self._offsets = [o for o in itertools.product((0, 1), repeat=ndim)]
        self._leaves = {(1, (x, y, z)) for z in range(self.nblk[2]) for y in range(self.nblk[1])
                        for x in range(self.nblk[0])}
        self._inner = set()
        self._finalize()

    def __getattr__(self, name):
        # key tables of a grid built from node arrays (regrid_native)
        if name in ("node_index", "_leaves", "_inner") and "levels" in self.__dict__:
            keys = [(int(lv), (int(c[0]), int(c[1]), int(c[2]))) for lv, c in zip(self.levels, self.coords)]
            self.node_index = {k: i for i, k in enumerate(keys)}
            self._leaves = {keys[i] for i in self.leaf_ids}
            self._inner = {keys[i] for i in np.nonzero(~self.is_leaf)[0]}
            return self.__dict__[name]
        raise AttributeError(name)

    # -- tree edits ----------------------------------------------------------
    def _extent(self, level):
        return tuple(self.nblk[d] * (2 ** (level - 1)) if d < self.ndim else 1 for d in range(3))

    def _children(self, level, c):
        out = []
        for o in self._offsets:
            cc = [2 * c[d] + (o[d] if d < len(o) else 0) if d < self.ndim else 0 for d in range(3)]
            out.append((level + 1, tuple(cc)))
        return out

    def _split(self, key):
        self._leaves.discard(key)
        self._inner.add(key)
        for ch in self._children(*key):
            self._leaves.add(ch)

    def refine(self, marker):
        """Refine every leaf below max_level for which marker(level, coords)
        is true, then restore the 2:1 balance."""
        for key in sorted(self._leaves):
            lev, c = key
            if lev < self.max_level and marker(lev, c):
                self._split(key)
        self._balance()
        self._finalize()

    def refine_levels(self, marker):
        """Refine level by level (1 .. max_level-1) with the same marker."""
        for lev in range(1, self.max_level):
            for key in sorted(k for k in self._leaves if k[0] == lev):
                if marker(lev, key[1]):
                    self._split(key)
            self._balance()
        self._finalize()

    def _neighbor(self, level, c, o):
        ext = self._extent(level)
        p = []
        for d in range(3):
            v = c[d] + (o[d] if d < self.ndim else 0)
            if d < self.ndim and (v < 0 or v >= ext[d]):
                if not self.periodic[d]:
                    return None
                v %= ext[d]
            p.append(v)
        return tuple(p)

    def _balance(self):
        offs = [o for o in itertools.product((-1, 0, 1), repeat=self.ndim) if any(o)]
        changed = True
        while changed:
            changed = False
            for key in sorted(self._leaves):
                lev, c = key
                if lev >= self.max_level:
                    continue
                need = False
                for o in offs:
                    o3 = tuple(o) + (0,) * (3 - self.ndim)
                    p = self._neighbor(lev, c, o3)
                    if p is None or (lev, p) not in self._inner:
                        continue
                    # children of the neighbour that touch this block
                    for ch_lev, ch in self._children(lev, p):
                        touch = True
                        for d in range(self.ndim):
                            co = ch[d] - 2 * p[d]
                            if (o3[d] == 1 and co != 0) or (o3[d] == -1 and co != 1):
                                touch = False
                        if touch and (ch_lev, ch) in self._inner:
                            need = True
                            break
                    if need:
                        break
                if need:
                    self._split(key)
                    changed = True

    # -- node arrays -----------------------------------------------------------
    def _finalize(self):
        nodes = sorted(self._leaves | self._inner, key=lambda k: (k[0], _morton(k[1])))
        self.node_index = {k: i for i, k in enumerate(nodes)}
        self.nblocks = len(nodes)
        self.levels = np.array([k[0] for k in nodes], dtype=np.int32)
        self.coords = np.array([k[1] for k in nodes], dtype=np.int32).reshape(-1, 3)
        self.is_leaf = np.array([k in self._leaves for k in nodes], dtype=bool)
        self.leaf_ids = np.nonzero(self.is_leaf)[0]
        self.parent = np.full(self.nblocks, -1, dtype=np.int32)
        for i, (lev, c) in enumerate(nodes):
            if lev > 1:
                self.parent[i] = self.node_index[(lev - 1, tuple(v // 2 if d < self.ndim else 0
                                                                 for d, v in enumerate(c)))]
        self.max_used_level = int(self.levels.max())
        self.delta_b = np.array([[self.delta1[d] / 2.0 ** (lv - 1) if d < self.ndim else 1.0 for d in range(3)]
                                 for lv in self.levels])

    @property
    def nleaves(self):
        return int(self.is_leaf.sum())

    @property
    def ncells(self):
        """Interior cells of the leaves (the zones a step advances)."""
        return self.nleaves * self.nb[0] * self.nb[1] * self.nb[2]

    def delta(self, level):
        return tuple(self.delta1[d] / 2.0 ** (level - 1) if d < self.ndim else 1.0 for d in range(3))

    def desc(self):
        g = abi.GridDesc()
        g.ndim = self.ndim
        g.nxb, g.nyb, g.nzb = self.nb
        g.nguard = self.nguard
        g.nblocks = self.nblocks
        for d in range(3):
            g.nblk_l1[d] = self.nblk[d]
            g.domain_lo[d] = self.lo[d]
            g.domain_hi[d] = self.hi[d]
        for f in range(6):
            g.bc[f] = self.bc[f]
        g.max_level = self.max_level
        self._keep = (np.ascontiguousarray(self.coords.reshape(-1)), np.ascontiguousarray(self.levels))
        g.block_coords = self._keep[0].ctypes.data_as(C.POINTER(C.c_int))
        g.block_level = self._keep[1].ctypes.data_as(C.POINTER(C.c_int))
        return g

    # -- UNK helpers (the same interface as UniformGrid) -------------------------
    def new_unk(self):
        return np.zeros((self.nblocks, self.nt[2], self.nt[1], self.nt[0], self.nunk), dtype=np.float64)

    @property
    def species(self):
        """UNK slice of the species and mass scalars."""
        return slice(NUNK, self.nunk)

    def interior(self, unk):
        g = self.ng
        return unk[:, g[2]:g[2] + self.nb[2], g[1]:g[1] + self.nb[1], g[0]:g[0] + self.nb[0], :]

    def cell_centers(self):
        out = []
        for d in range(3):
            n = self.nb[d]
            c = self.coords[:, d][:, None] * n + (np.arange(n) + 0.5)[None, :]
            c = self.lo[d] + c * self.delta_b[:, d][:, None] if d < self.ndim else np.zeros_like(c, dtype=np.float64)
            shape = [self.nblocks, 1, 1, 1]
            shape[3 - d] = n
            out.append(np.broadcast_to(c.reshape(shape), (self.nblocks, self.nb[2], self.nb[1], self.nb[0])))
        return out

    def cell_edges(self, d):
        n = self.nb[d]
        lft = self.coords[:, d][:, None] * n + np.arange(n)[None, :]
        xl = self.lo[d] + lft * self.delta_b[:, d][:, None]
        xr = self.lo[d] + (lft + 1) * self.delta_b[:, d][:, None]
        shape = [self.nblocks, 1, 1, 1]
        shape[3 - d] = n
        full = (self.nblocks, self.nb[2], self.nb[1], self.nb[0])
        return np.broadcast_to(xl.reshape(shape), full), np.broadcast_to(xr.reshape(shape), full)

    def cell_volumes(self):
        v = np.prod(self.delta_b[:, :self.ndim], axis=1)
        return v

    def composite(self, unk, var, level=None):
        """One variable of the leaves on a uniform (nz, ny, nx) image at
        `level` (default: the finest used level); coarse leaves are
        injected (repeated), finer leaves averaged."""
        level = self.max_used_level if level is None else level
        ext = self._extent(level)
        shape = tuple(ext[d] * self.nb[d] if d < self.ndim else 1 for d in (2, 1, 0))
        out = np.zeros(shape)
        it = self.interior(unk)[..., VAR[var]]
        for b in self.leaf_ids:
            lv = self.levels[b]
            f = 2 ** (level - lv) if level >= lv else None
            data = it[b]
            if f is None:
                r = 2 ** (lv - level)
                sh = (data.shape[0] // (r if self.ndim > 2 else 1), r if self.ndim > 2 else 1,
                      data.shape[1] // r, r, data.shape[2] // r, r)
                data = data.reshape(sh).mean(axis=(1, 3, 5))
                f = 1
                scale = 1.0 / r
            else:
                scale = float(f)
                for ax in range(3):
                    if (2 - ax) < self.ndim:
                        data = np.repeat(data, f, axis=ax)
            o = [int(self.coords[b, d] * self.nb[d] * scale) if d < self.ndim else 0 for d in range(3)]
            out[o[2]:o[2] + data.shape[0], o[1]:o[1] + data.shape[1], o[0]:o[0] + data.shape[2]] = data
        return out


def indicator_refiner(grid, field, threshold):
    """Marker for AmrGrid.refine_levels: refine a block where the
    dimensionless density gradient |grad rho| * dx / rho of `field` (a
    function of cell-centre coordinates), sampled at the block's own
    resolution with one extra ring of cells, exceeds `threshold`."""
    def marker(level, c):
        dx = grid.delta(level)
        ax = []
        for d in range(3):
            if d < grid.ndim:
                n = grid.nb[d]
                ax.append(grid.lo[d] + (c[d] * n + np.arange(-1, n + 1) + 0.5) * dx[d])
            else:
                ax.append(np.array([0.0]))
        Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        rho = field(X, Y, Z)
        inner = tuple(slice(1, -1) if (2 - a) < grid.ndim else slice(None) for a in range(3))
        ind = np.zeros_like(rho[inner])
        for d in range(grid.ndim):
            a = 2 - d
            hi = list(inner); lo = list(inner)
            hi[a] = slice(2, None); lo[a] = slice(None, -2)
            ind = ind + (0.5 * (rho[tuple(hi)] - rho[tuple(lo)])) ** 2
        return bool(np.max(np.sqrt(ind) / rho[inner]) > threshold)
    return marker


def four_quadrant_refinement_field(seed=2024, modes=12, width=0.004):
    """Seeded smoothed density used to build the benchmark hierarchy: the
    four-quadrant densities blended across x = 0.5 and y = 0.5 by tanh
    profiles of the given width, times 1 + a sum of `modes` seeded Fourier
    modes (wave numbers 1..8 per axis, amplitudes 0.02..0.06, numpy PCG64)."""
    rng = np.random.default_rng(seed)
    kx = rng.integers(1, 9, modes)
    ky = rng.integers(1, 9, modes)
    ph = rng.uniform(0, 2 * np.pi, modes)
    am = rng.uniform(0.02, 0.06, modes)

    def field(X, Y, Z):
        sx = 0.5 * (1 + np.tanh((X - 0.5) / width))
        sy = 0.5 * (1 + np.tanh((Y - 0.5) / width))
        r = (1 - sx) * (1 - sy) * 0.138 + sx * (1 - sy) * 0.5323 + (1 - sx) * sy * 0.5323 + sx * sy * 1.5
        pert = sum(am[k] * np.sin(2 * np.pi * (kx[k] * X + ky[k] * Y) + ph[k]) for k in range(modes))
        return r * (1 + pert)
    return field


def four_quadrant_hierarchy(nb=16, nblk=32, max_level=4, threshold=0.0035, seed=2024, bc="outflow"):
    """The batched AMR benchmark hierarchy: [0,1]^2, nblk^2 root blocks of
    nb^2 cells, max_level levels, refined level by level where the
    dimensionless density gradient of four_quadrant_refinement_field
    exceeds `threshold` (defaults: 19,456 leaf blocks of 16^2 on levels
    1-4, about 5.0e6 leaf zones)."""
    g = AmrGrid(2, (nb, nb), (nblk, nblk), max_level, bc=bc)
    g.refine_levels(indicator_refiner(g, four_quadrant_refinement_field(seed), threshold))
    return g


# -- refinement and derefinement (Grid_markRefineDerefine, gr_updateRefinement) --

def mark_refine_derefine(grid, errors, refine_cutoff, derefine_cutoff, max_refine=None):
    """Refine / derefine flags of every node from the estimator's errors,
    one array per refinement variable (Grid/GridMain/AMR/
    Grid_markRefineDerefine.F90 and paramesh4/gr_markRefineDerefine.F90):
    per variable, a leaf is marked for derefinement when it is not marked
    for refinement or to stay and both its error and its parent's are at or
    below the derefine cutoff; any node above the refine cutoff is marked
    for refinement (not above max_refine); a leaf above the derefine cutoff
    or under a parent above it stays.  Only leaves keep their marks.
    refine_cutoff / derefine_cutoff: scalars or one value per variable."""
    n = grid.nblocks
    nv = len(errors)
    rc = np.broadcast_to(np.asarray(refine_cutoff, dtype=np.float64), (nv,))
    dc = np.broadcast_to(np.asarray(derefine_cutoff, dtype=np.float64), (nv,))
    max_refine = grid.max_level if max_refine is None else int(max_refine)
    refine = np.zeros(n, dtype=bool)
    derefine = np.zeros(n, dtype=bool)
    stay = np.zeros(n, dtype=bool)
    leaf = grid.is_leaf
    top = grid.levels >= max_refine
    for v in range(nv):
        err = np.asarray(errors[v], dtype=np.float64)
        err_par = np.where(grid.parent >= 0, err[np.maximum(grid.parent, 0)], 0.0)
        # the per-block rules, all blocks at once (each block's marks depend
        # only on its own and its parent's error and its earlier marks)
        derefine = leaf & ~refine & ~stay & (err <= dc[v]) & (err_par <= dc[v])
        up = err > rc[v]
        derefine &= ~up
        refine |= up
        stay |= (leaf & (err > dc[v])) | (err_par > dc[v])
        refine &= ~top
    refine &= leaf
    derefine &= leaf
    return refine, derefine


def _clone(grid):
    g = copy.copy(grid)
    g._leaves = set(grid._leaves)
    g._inner = set(grid._inner)
    return g


def _grid_from_nodes(template, levels, coords, parent):
    """An AmrGrid with the given nodes (ordered by level and Morton index)."""
    g = copy.copy(template)
    g.nblocks = len(levels)
    g.levels = np.ascontiguousarray(levels, dtype=np.int32)
    g.coords = np.ascontiguousarray(np.asarray(coords, dtype=np.int32).reshape(-1, 3))
    g.parent = np.ascontiguousarray(parent, dtype=np.int32)
    leaf = np.ones(g.nblocks, dtype=bool)
    leaf[g.parent[g.parent >= 0]] = False
    g.is_leaf = leaf
    g.leaf_ids = np.nonzero(leaf)[0]
    # the key tables of the Python tree code are built on first use
    for a in ("node_index", "_leaves", "_inner"):
        g.__dict__.pop(a, None)
    g.max_used_level = int(g.levels.max())
    scale = np.ldexp(1.0, 1 - g.levels.astype(np.int64))
    g.delta_b = np.stack([g.delta1[d] * scale if d < g.ndim else np.ones(g.nblocks) for d in range(3)], axis=1)
    return g


def regrid_native(grid, refine, derefine, min_level=1):
    """regrid() by the library's tree code (flash_hy_refine_tree)."""
    lib = abi.load_library()
    gd = grid.desc()
    r = np.ascontiguousarray(np.asarray(refine, dtype=np.uint8))
    d = np.ascontiguousarray(np.asarray(derefine, dtype=np.uint8))
    cap = grid.nblocks + (2 ** grid.ndim) * int(grid.is_leaf.sum()) + 8
    out = [np.empty(cap, dtype=np.int32) for _ in range(5)]
    coords = np.empty(3 * cap, dtype=np.int32)
    n = C.c_int()
    pi = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    st = lib.flash_hy_refine_tree(C.byref(gd), r.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p),
                                  int(min_level), cap, C.byref(n), pi(out[0]), pi(coords), pi(out[1]), pi(out[2]),
                                  pi(out[3]))
    if st:
        raise RuntimeError(f"flash_hy_refine_tree status {st:#x}")
    n = n.value
    g = _grid_from_nodes(grid, out[0][:n], coords[:3 * n], out[1][:n])
    return g, out[2][:n].copy(), out[3][:n].copy()


def regrid(grid, refine, derefine, min_level=1):
    """The hierarchy after the marked refinements and derefinements, with
    PARAMESH's rules: a marked leaf below max_level is split and refinement
    spreads to keep neighbours (diagonals included) within one level; a
    parent's children are removed when all of them are leaves marked for
    derefinement that were not refined, the parent is above min_level - 1
    and no neighbour of the parent would be two levels finer.  Returns
    (new grid, src, how): for every new node, how = 0 copies old node src,
    1 is a new child of old leaf src (prolonged), 2 is old parent src made a
    leaf (derefined)."""
    old = grid
    g = _clone(old)
    key_of = {i: k for k, i in old.node_index.items()}
    for b in np.nonzero(np.asarray(refine) & old.is_leaf)[0]:
        key = key_of[int(b)]
        if key[0] < g.max_level:
            g._split(key)
    g._balance()
    # derefinement, decided on the tree after refinement: candidates are the
    # parents all of whose children are unrefined marked leaves; a candidate
    # is dropped while a neighbour's child touching it stays refined (is not
    # a candidate itself), until the set no longer changes
    offs = [o for o in itertools.product((-1, 0, 1), repeat=g.ndim) if any(o)]
    dmark = {key_of[int(b)] for b in np.nonzero(np.asarray(derefine) & old.is_leaf)[0]}
    cand = set()
    for pkey in old._inner:
        lev, pc = pkey
        if lev >= min_level and all(k in g._leaves and k in dmark for k in g._children(lev, pc)):
            cand.add(pkey)

    def blocked(pkey):
        lev, pc = pkey
        for o in offs:
            o3 = tuple(o) + (0,) * (3 - g.ndim)
            nkey = g._neighbor(lev, pc, o3)
            if nkey is None or (lev, nkey) not in g._inner:
                continue
            for ch in g._children(lev, nkey):
                touch = all(not ((o3[d] == 1 and ch[1][d] - 2 * nkey[d] != 0) or
                                 (o3[d] == -1 and ch[1][d] - 2 * nkey[d] != 1)) for d in range(g.ndim))
                if touch and ch in g._inner and ch not in cand:
                    return True
        return False

    changed = True
    while changed:
        changed = False
        for pkey in sorted(cand):
            if blocked(pkey):
                cand.discard(pkey)
                changed = True
    merge = sorted(cand)
    for pkey in merge:
        for k in g._children(*pkey):
            g._leaves.discard(k)
        g._inner.discard(pkey)
        g._leaves.add(pkey)
    g._finalize()
    new_key = {i: k for k, i in g.node_index.items()}
    src = np.empty(g.nblocks, dtype=np.int32)
    how = np.empty(g.nblocks, dtype=np.int32)
    for q in range(g.nblocks):
        key = new_key[q]
        if key in old.node_index:
            src[q] = old.node_index[key]
            how[q] = 2 if (key in old._inner and key in g._leaves) else 0
        else:
            lev, c = key
            pkey = (lev - 1, tuple(v // 2 if d < g.ndim else 0 for d, v in enumerate(c)))
            if pkey not in old._leaves:
                raise RuntimeError("regrid created a node two levels below the old tree")
            src[q] = old.node_index[pkey]
            how[q] = 1
    return g, src, how


def update_refinement(h, grid, refine_vars=("dens", "pres"), refine_cutoff=0.8, derefine_cutoff=0.2,
                      refine_filter=0.01, min_level=1, timings=None):
    """Grid_markRefineDerefine + Grid_updateRefinement on a device context:
    the estimator of every refinement variable, the marks and the new tree
    on the device (flash_hy_mark_refine_tree), the new grid's descriptors on
    the host, the data of the new tree on the device (flash_hy_regrid).
    Returns (context, grid): the old ones when nothing changes, else a new
    context (the old one is closed) for the new grid.  `timings`, a dict,
    receives the seconds of each phase."""
    import time
    t0 = time.perf_counter()
    lev, coords, par, src, how = h.mark_refine_tree(refine_vars, refine_filter, refine_cutoff, derefine_cutoff,
                                                    min_level=min_level)
    t1 = time.perf_counter()
    changed = len(lev) != grid.nblocks or np.any(how != 0)
    if changed:
        g2 = _grid_from_nodes(grid, lev, coords, par)
        t2 = time.perf_counter()
        h2 = h.regrid(g2, src, how)
        h.close()
        h, grid = h2, g2
    else:
        t2 = time.perf_counter()
    t3 = time.perf_counter()
    if timings is not None:
        timings.update(mark_and_tree_s=t1 - t0, grid_s=t2 - t1, data_s=t3 - t2,
                       refined=int(np.count_nonzero(how == 1)), derefined=int(np.count_nonzero(how == 2)),
                       changed=bool(changed))
    return h, grid
