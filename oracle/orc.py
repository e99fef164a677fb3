"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, always as the checker.  The oracle library is built by
``oracle/Makefile`` (``make -C oracle``).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from flash5_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc_hy.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, G = C.POINTER(abi.Params), C.POINTER(abi.GridDesc)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_fill_guardcells.argtypes = [P, G, dp]
        L.orc_eos_interior.argtypes = [P, G, dp]
        L.orc_hydro.argtypes = [P, G, dp, C.c_double, C.c_double, C.c_double, C.c_int, ip]
        L.orc_compute_dt.argtypes = [P, G, dp, dp, ip]
        L.orc_hllc.argtypes = [P, C.c_int, dp, dp, dp]
        L.orc_exact_flux.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_int, dp, ip]
        L.orc_star_state.argtypes = [C.c_double] * 8 + [C.c_double, C.c_int, dp, dp, ip]
        L.orc_estimate_error.argtypes = [C.c_void_p, C.c_void_p, dp, C.c_int, C.c_double, dp]
        L.orc_amr_regrid.argtypes = [C.c_void_p, C.c_void_p, dp, C.c_void_p, dp, ip, ip]
        L.orc_two_rarefaction_guess.argtypes = [C.c_double] * 7
        L.orc_two_rarefaction_guess.restype = C.c_double
        L.orc_star_batch.argtypes = [C.c_long] + [dp] * 8 + [C.c_double, C.c_int, dp, dp, ip, ip]
        L.orc_amr_fill_guardcells.argtypes = [P, G, dp]
        L.orc_amr_hydro.argtypes = [P, G, dp, C.c_double, C.c_double, C.c_double]
        L.orc_amr_compute_dt.argtypes = [P, G, dp, dp, ip]
        L.orc_amr_restrict.argtypes = [P, G, dp]
        L.orc_block_fluxes.argtypes = [P, G, dp, C.c_int, C.c_double, dp]
        _lib = L
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FLASH-like driver over host UNK arrays: eos_init, hydro step, dt.
    Grids with max_level > 1 (AmrGrid) use the AMR restatement."""

    def __init__(self, params, grid):
        from flash5_b200 import abi
        self.p = abi.with_species(params, grid)
        self.grid = grid
        self.g = grid.desc()
        self.amr = self.g.max_level > 1

    def eos_init(self, unk):
        st = lib().orc_eos_interior(C.byref(self.p), C.byref(self.g), _dp(unk))
        assert st == 0, st
        if self.amr:
            st = lib().orc_amr_restrict(C.byref(self.p), C.byref(self.g), _dp(unk))
            assert st == 0, st
        return unk

    def fill_guardcells(self, unk):
        if self.amr:
            return lib().orc_amr_fill_guardcells(C.byref(self.p), C.byref(self.g), _dp(unk))
        return lib().orc_fill_guardcells(C.byref(self.p), C.byref(self.g), _dp(unk))

    def hydro(self, unk, sim_time, dt, dt_old, blocks=None):
        if self.amr:
            assert blocks is None
            return lib().orc_amr_hydro(C.byref(self.p), C.byref(self.g), _dp(unk), sim_time, dt, dt_old)
        if blocks is None:
            return lib().orc_hydro(C.byref(self.p), C.byref(self.g), _dp(unk), sim_time, dt, dt_old, 0, None)
        bl = np.ascontiguousarray(blocks, dtype=np.int32)
        return lib().orc_hydro(C.byref(self.p), C.byref(self.g), _dp(unk), sim_time, dt, dt_old, len(bl),
                               bl.ctypes.data_as(C.POINTER(C.c_int)))

    def estimate_error(self, unk, var="dens", refine_filter=0.01):
        """gr_estimateError on a copy of unk (guard cells filled there)."""
        from flash5_b200 import abi
        u = np.ascontiguousarray(unk.copy())
        err = np.zeros(self.grid.nblocks, dtype=np.float64)
        st = lib().orc_estimate_error(C.byref(self.p), C.byref(self.g), _dp(u), abi.REFVAR[var],
                                      float(refine_filter), _dp(err))
        assert st == 0, st
        return err

    def regrid(self, unk, new_grid, src, how):
        """gr_updateRefinement's data movement on host UNK arrays: the UNK of
        new_grid (amr.regrid's tree) from unk (whose guard cells are
        refilled)."""
        out = new_grid.new_unk()
        gn = new_grid.desc()
        s = np.ascontiguousarray(src, dtype=np.int32)
        w = np.ascontiguousarray(how, dtype=np.int32)
        st = lib().orc_amr_regrid(C.byref(self.p), C.byref(self.g), _dp(unk), C.byref(gn), _dp(out),
                                  s.ctypes.data_as(C.POINTER(C.c_int)), w.ctypes.data_as(C.POINTER(C.c_int)))
        assert st == 0, st
        return out

    def amr_hydro(self, unk, sim_time, dt, dt_old):
        """The AMR step on any grid (max_level 1 included)."""
        return lib().orc_amr_hydro(C.byref(self.p), C.byref(self.g), _dp(unk), sim_time, dt, dt_old)

    def block_fluxes(self, unk, blk, dt):
        """Face fluxes of block blk, [ndim][faces][NFLUXES] in FLASH's flux
        layout (NFLUXES = 8 + species + mass scalars)."""
        nb = self.grid.nb
        nf = (nb[0] + 1) * nb[1] * nb[2]
        nsp = getattr(self.grid, "nspecies", 0) + getattr(self.grid, "nmass_scalars", 0)
        out = np.zeros((self.grid.ndim, nf, 8 + nsp))
        st = lib().orc_block_fluxes(C.byref(self.p), C.byref(self.g), _dp(unk), blk, dt, _dp(out))
        return st, out

    def compute_dt(self, unk):
        """(status, dt, loc): loc = (i, j, k, level, meshMe, block), FLASH's
        dtMinLoc (meshMe = 0 for one rank) and the 0-based block."""
        dt = C.c_double()
        loc = (C.c_int * 6)()
        f = lib().orc_amr_compute_dt if self.amr else lib().orc_compute_dt
        st = f(C.byref(self.p), C.byref(self.g), _dp(unk), C.byref(dt), loc)
        return st, dt.value, tuple(loc)


def hllc(params, dirn, VL, VR):
    VL = np.ascontiguousarray(VL, dtype=np.float64)
    VR = np.ascontiguousarray(VR, dtype=np.float64)
    F = np.zeros(6)
    st = lib().orc_hllc(C.byref(params), dirn, _dp(VL), _dp(VR), _dp(F))
    return st, F


def exact_flux(dirn, VL, VR, gamma, tol=1e-12, max_iter=50):
    """Godunov flux of the exact solution (6 slots as hllc); (F, status, evaluations)."""
    VL = np.ascontiguousarray(VL, dtype=np.float64)
    VR = np.ascontiguousarray(VR, dtype=np.float64)
    F = np.zeros(6)
    it = C.c_int()
    st = lib().orc_exact_flux(dirn, _dp(VL), _dp(VR), gamma, tol, max_iter, _dp(F), C.byref(it))
    return F, st, it.value


def star_state(dl, ul, pl, dr, ur, pr, gamma, p0=0.0, tol=1e-12, max_iter=50):
    ps, us, it = C.c_double(), C.c_double(), C.c_int()
    st = lib().orc_star_state(dl, ul, pl, dr, ur, pr, gamma, p0, tol, max_iter, C.byref(ps), C.byref(us),
                              C.byref(it))
    return st, ps.value, us.value, it.value


def star_batch(dl, ul, pl, dr, ur, pr, gam, p0=None, tol=1e-12, max_iter=50):
    n = len(dl)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dl, ul, pl, dr, ur, pr, gam)]
    p0a = None if p0 is None else np.ascontiguousarray(p0, dtype=np.float64)
    ps, us = np.zeros(n), np.zeros(n)
    it, st = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib().orc_star_batch(n, *[_dp(a) for a in arrs], None if p0a is None else _dp(p0a), tol, max_iter,
                         _dp(ps), _dp(us), it.ctypes.data_as(C.POINTER(C.c_int)),
                         st.ctypes.data_as(C.POINTER(C.c_int)))
    return ps, us, it, st


def two_rarefaction_guess(dl, ul, pl, dr, ur, pr, gamma):
    return lib().orc_two_rarefaction_guess(dl, ul, pl, dr, ur, pr, gamma)
