"""Block-structured grid helpers: descriptors and FLASH UNK arrays.

A uniform grid of ``nblk`` blocks per axis, each of ``nb`` interior cells,
with FLASH's NGUARD = 4 guard layers in the host UNK array
(unsplit/Config:209-211).  Host UNK uses the default FLASH ordering
unk(var, i, j, k, blk) with variables in the alphabetical +uhd/gamma-EOS
order (bin/unitCfg.py:713-714), i.e. a C array of shape
(nblocks, nzt, nyt, nxt, nunk), nunk = NUNK + species + mass scalars (the
species and mass scalars follow the property variables, as SPECIES_BEGIN ..
MASS_SCALARS_END in Flash.h).
"""
import ctypes as C
import numpy as np

from . import abi

NGUARD = 4
NUNK = len(abi.FLASH_UHD_VARS)
VAR = {n: i for i, n in enumerate(abi.FLASH_UHD_VARS)}


class UniformGrid:
    def __init__(self, ndim, nb, nblk, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), bc="outflow", order="lex",
                 nguard=NGUARD, nspecies=0, nmass_scalars=0):
        self.ndim = ndim
        self.nspecies, self.nmass_scalars = int(nspecies), int(nmass_scalars)
        self.nunk = NUNK + self.nspecies + self.nmass_scalars
        nb = tuple(nb) + (1,) * (3 - len(nb))
        nblk = tuple(nblk) + (1,) * (3 - len(nblk))
        self.nb = tuple(nb[d] if d < ndim else 1 for d in range(3))
        self.nblk = tuple(nblk[d] if d < ndim else 1 for d in range(3))
        self.lo = tuple(lo)
        self.hi = tuple(hi)
        if isinstance(bc, str):
            bc = [bc] * 6
        code = {"outflow": abi.BC_OUTFLOW, "periodic": abi.BC_PERIODIC, "reflecting": abi.BC_REFLECTING}
        self.bc = [code[b] if isinstance(b, str) else int(b) for b in bc]
        self.bc += [abi.BC_OUTFLOW] * (6 - len(self.bc))      # faces of absent dimensions
        coords = [(bx, by, bz) for bz in range(self.nblk[2]) for by in range(self.nblk[1]) for bx in range(self.nblk[0])]
        if order == "morton":
            def key(c):
                k = 0
                for bit in range(16):
                    for d in range(3):
                        k |= ((c[d] >> bit) & 1) << (3 * bit + d)
                return k
            coords.sort(key=key)
        self.coords = np.array(coords, dtype=np.int32)
        self.nblocks = len(coords)
        self.levels = np.ones(self.nblocks, dtype=np.int32)
        self.nguard = nguard
        self.ng = (nguard, nguard if ndim > 1 else 0, nguard if ndim > 2 else 0)
        self.nt = tuple(self.nb[d] + 2 * self.ng[d] for d in range(3))
        self.delta = tuple((self.hi[d] - self.lo[d]) / (self.nblk[d] * self.nb[d]) if d < ndim else 1.0
                           for d in range(3))

    @property
    def ncells(self):
        return self.nblocks * self.nb[0] * self.nb[1] * self.nb[2]

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
        g.max_level = 1
        self._keep = (np.ascontiguousarray(self.coords.reshape(-1)), np.ascontiguousarray(self.levels))
        g.block_coords = self._keep[0].ctypes.data_as(C.POINTER(C.c_int))
        g.block_level = self._keep[1].ctypes.data_as(C.POINTER(C.c_int))
        return g

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
        """Per-block arrays (x, y, z) of interior cell centres, each of shape
        (nblocks, nzb, nyb, nxb)."""
        out = []
        for d in range(3):
            n = self.nb[d]
            loc = (np.arange(n) + 0.5)
            c = self.coords[:, d][:, None] * n + loc[None, :]
            c = self.lo[d] + c * self.delta[d] if d < self.ndim else np.zeros_like(c, dtype=np.float64)
            shape = [self.nblocks, 1, 1, 1]
            shape[3 - d] = n
            out.append(np.broadcast_to(c.reshape(shape), (self.nblocks, self.nb[2], self.nb[1], self.nb[0])))
        return out

    def cell_edges(self, d):
        n = self.nb[d]
        lft = self.coords[:, d][:, None] * n + np.arange(n)[None, :]
        xl = self.lo[d] + lft * self.delta[d]
        xr = self.lo[d] + (lft + 1) * self.delta[d]
        shape = [self.nblocks, 1, 1, 1]
        shape[3 - d] = n
        full = (self.nblocks, self.nb[2], self.nb[1], self.nb[0])
        return np.broadcast_to(xl.reshape(shape), full), np.broadcast_to(xr.reshape(shape), full)

    def to_global(self, unk, var):
        """Assemble one variable's interiors into a global (nz, ny, nx) array."""
        it = self.interior(unk)[..., VAR[var]]
        nx, ny, nz = (self.nblk[d] * self.nb[d] for d in range(3))
        out = np.empty((nz, ny, nx))
        for b, (bx, by, bz) in enumerate(self.coords):
            out[bz * self.nb[2]:(bz + 1) * self.nb[2], by * self.nb[1]:(by + 1) * self.nb[1],
                bx * self.nb[0]:(bx + 1) * self.nb[0]] = it[b]
        return out
