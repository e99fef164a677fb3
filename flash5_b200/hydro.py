"""Host-side mirror of FLASH5's Hydro interface over the CUDA C-ABI.

``Hydro`` mirrors ``Hydro_init`` / ``Hydro(simTime, dt, dtOld, sweepOrder)``
/ ``Hydro_computeDt`` (source/physics/Hydro/Hydro_interface.F90:12-137,
HydroMain/unsplit/Hydro.F90:6-343) and the FLASH4-style
``Hydro(blockCount, blockList, timeEndAdv, dt, dtOld, sweepOrder)``.
Errors come back as ``HydroError`` with the C-ABI status bits; FLASH aborts
the run in the same situations (Driver_abortFlash).

Blocks are numbered here as numpy indexes the grid's block axis (0-based);
the C ABI takes FLASH's 1-based block IDs, and this module converts.
"""
import ctypes as C

import numpy as np

from . import abi


class HydroError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        names = [n for n in dir(abi) if n.startswith("ERR_") and getattr(abi, n) & status]
        super().__init__(f"flash_hy status {status:#x} {names} {msg}")


class Hydro:
    """One device context holding the block store of a grid."""

    def __init__(self, params, grid, device=0):
        self.lib = abi.load_library()
        self.device = device
        params = abi.with_species(params, grid)
        self.params = params
        self.grid = grid
        self._gdesc = grid.desc()
        self.ctx = C.c_void_p()
        st = self.lib.flash_hy_create(C.byref(params), C.byref(self._gdesc), device, C.byref(self.ctx))
        if st:
            msg = self.last_error() if self.ctx else ""
            if self.ctx:
                self.lib.flash_hy_destroy(self.ctx)
                self.ctx = C.c_void_p()
            raise HydroError(st, msg)
        self.varmap = abi.flash_varmap(params.nspecies + params.nmass_scalars)

    # -- lifecycle -------------------------------------------------------
    def close(self):
        if self.ctx:
            self.lib.flash_hy_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self):
        buf = C.create_string_buffer(512)
        self.lib.flash_hy_last_error(self.ctx, buf, 512)
        return buf.value.decode()

    def _check(self, st):
        if st:
            raise HydroError(st, self.last_error())

    # -- Grid data --------------------------------------------------------
    def upload(self, unk, layout=abi.LAYOUT_VAR_FASTEST):
        unk = np.ascontiguousarray(unk, dtype=np.float64)
        self._check(self.lib.flash_hy_upload(self.ctx, unk.ctypes.data_as(C.POINTER(C.c_double)), layout,
                                             unk.shape[-1] if layout == abi.LAYOUT_VAR_FASTEST else unk.shape[1],
                                             C.byref(self.varmap)))

    def download(self, unk, layout=abi.LAYOUT_VAR_FASTEST):
        assert unk.dtype == np.float64 and unk.flags.c_contiguous
        self._check(self.lib.flash_hy_download(self.ctx, unk.ctypes.data_as(C.POINTER(C.c_double)), layout,
                                               unk.shape[-1] if layout == abi.LAYOUT_VAR_FASTEST else unk.shape[1],
                                               C.byref(self.varmap)))
        return unk

    # -- the hot path -----------------------------------------------------
    def __call__(self, simTime, dt, dtOld, sweepOrder=0):
        """Hydro(simTime, dt, dtOld, sweepOrder): enqueue one step (async)."""
        self._check(self.lib.flash_hy_step(self.ctx, simTime, dt, dtOld, sweepOrder))

    def step_blocks(self, blockList, timeEndAdv, dt, dtOld, sweepOrder=0):
        """FLASH4's Hydro(blockCount, blockList, ...) on the blocks of
        blockList (0-based block indices)."""
        bl = _flash_ids(blockList)
        self._check(self.lib.flash_hy_step_blocks(self.ctx, len(bl), bl.ctypes.data_as(C.POINTER(C.c_int)),
                                                  timeEndAdv, dt, dtOld, sweepOrder))

    # -- split step: hy_computeFluxes / hy_updateSolution ------------------
    def compute_fluxes(self, blockList, dt, flags=abi.UPDATE_NONE):
        bl = _flash_ids(blockList)
        self._check(self.lib.flash_hy_compute_fluxes(self.ctx, len(bl), bl.ctypes.data_as(C.POINTER(C.c_int)), dt,
                                                     flags))

    def get_fluxes(self, block, dir):
        """Fluxes of one block in direction dir (1..ndim): [faces, NFLUXES]
        in FLASH's flx(NFLUXES, i, j, k) order, NFLUXES = 8 hydro fluxes +
        the species and mass-scalar fluxes."""
        nb = self.grid.nb
        nsp = getattr(self.grid, "nspecies", 0) + getattr(self.grid, "nmass_scalars", 0)
        out = np.zeros(((nb[0] + 1) * nb[1] * nb[2], 8 + nsp))
        self._check(self.lib.flash_hy_get_fluxes(self.ctx, int(block) + 1, dir,
                                                 out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def put_fluxes(self, block, dir, flx):
        flx = np.ascontiguousarray(flx, dtype=np.float64)
        nb = self.grid.nb
        nsp = getattr(self.grid, "nspecies", 0) + getattr(self.grid, "nmass_scalars", 0)
        if flx.shape != ((nb[0] + 1) * nb[1] * nb[2], 8 + nsp):
            raise ValueError(f"fluxes must have shape [faces, {8 + nsp}], got {flx.shape}")
        self._check(self.lib.flash_hy_put_fluxes(self.ctx, int(block) + 1, dir,
                                                 flx.ctypes.data_as(C.POINTER(C.c_double))))

    def update_solution(self, blockList, dt):
        bl = _flash_ids(blockList)
        self._check(self.lib.flash_hy_update_solution(self.ctx, len(bl), bl.ctypes.data_as(C.POINTER(C.c_int)), dt))

    def compute_dt(self):
        """Hydro_computeDt + the MINLOC reduction: (dt, (i, j, k, level,
        meshMe, block)) -- FLASH's dtMinLoc, then the 0-based block of the
        limiting cell (flash_hy_dt_block)."""
        dt = C.c_double()
        loc = (C.c_int * 5)()
        self._check(self.lib.flash_hy_compute_dt(self.ctx, C.byref(dt), loc))
        bid = C.c_int()
        self._check(self.lib.flash_hy_dt_block(self.ctx, C.byref(bid)))
        return dt.value, tuple(loc) + (bid.value - 1,)

    def set_mesh_me(self, rank):
        """hy_meshMe: the rank reported in the dt location."""
        self._check(self.lib.flash_hy_set_mesh_me(self.ctx, int(rank)))

    def sync(self):
        self._check(self.lib.flash_hy_sync(self.ctx))

    def export_state(self, torch):
        """The device state as a [5, ncells] float64 CUDA tensor (dens, velx,
        vely, velz, eint; blocks in descriptor order, each block's interior
        x fastest), copied on the context's stream and synchronised."""
        n = self.grid.nblocks * self.grid.nb[0] * self.grid.nb[1] * self.grid.nb[2]
        out = torch.empty((5, n), dtype=torch.float64, device=torch.device("cuda", self.device))
        torch.cuda.current_stream(out.device).synchronize()
        self._check(self.lib.flash_hy_export_state(self.ctx, C.c_void_p(out.data_ptr())))
        self.sync()
        return out

    # -- refinement ---------------------------------------------------------
    def estimate_error(self, var="dens", refine_filter=0.01):
        """gr_estimateError: Lohner's estimator of `var` for every block
        (numpy array indexed by block; 0 for ghost blocks of a rank's share)."""
        err = np.zeros(self.grid.nblocks, dtype=np.float64)
        self._check(self.lib.flash_hy_estimate_error(self.ctx, abi.REFVAR[var], float(refine_filter),
                                                      err.ctypes.data_as(C.POINTER(C.c_double))))
        return err

    def mark_refine_tree(self, refine_vars, refine_filter, refine_cutoff, derefine_cutoff, max_refine=None,
                         min_level=1):
        """Grid_markRefineDerefine and the tree of a regrid on the device
        (flash_hy_mark_refine_tree): the estimator, FLASH's marks and
        PARAMESH's tree rules.  Returns (levels, coords [n, 3], parent, src,
        how) of the new tree, ordered by level and Morton index."""
        nv = len(refine_vars)
        vars_ = (C.c_int * nv)(*[abi.REFVAR[v] for v in refine_vars])
        rc = (C.c_double * nv)(*np.broadcast_to(np.asarray(refine_cutoff, dtype=np.float64), (nv,)))
        dc = (C.c_double * nv)(*np.broadcast_to(np.asarray(derefine_cutoff, dtype=np.float64), (nv,)))
        g = self.grid
        cap = g.nblocks + (2 ** g.ndim) * int(g.is_leaf.sum()) + 8
        mr = g.max_level if max_refine is None else int(max_refine)
        lev, par, src, how = (np.empty(cap, dtype=np.int32) for _ in range(4))
        coords = np.empty(3 * cap, dtype=np.int32)
        n = C.c_int()
        pi = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self.lib.flash_hy_mark_refine_tree(self.ctx, nv, vars_, float(refine_filter), rc, dc, mr,
                                                       int(min_level), cap, C.byref(n), pi(lev), pi(coords), pi(par),
                                                       pi(src), pi(how)))
        n = n.value
        return lev[:n].copy(), coords[:3 * n].reshape(n, 3).copy(), par[:n].copy(), src[:n].copy(), how[:n].copy()

    def regrid(self, new_grid, src, how):
        """gr_updateRefinement's data movement: a new context for new_grid
        (amr.regrid's tree) filled from this one; this context is left as it
        was (its parents restricted)."""
        h = Hydro(self.params, new_grid, device=self.device)
        s = np.ascontiguousarray(src, dtype=np.int32)
        w = np.ascontiguousarray(how, dtype=np.int32)
        st = self.lib.flash_hy_regrid(self.ctx, h.ctx, len(s), s.ctypes.data_as(C.POINTER(C.c_int)),
                                      w.ctypes.data_as(C.POINTER(C.c_int)))
        if st:
            msg = h.last_error() or self.last_error()
            h.close()
            raise HydroError(st, msg)
        return h

    # -- launch shapes ----------------------------------------------------
    @property
    def tuning(self):
        """Launch shape of the step (dict): threads per CTA of the step's
        kernels, blocks per CTA of the mixed 3D direction kernels (mx_runs)
        and the mixed path's sweep order (mx_sweep, abi.SWEEP_XYZ or
        abi.SWEEP_ZYX)."""
        t = abi.Tuning()
        self._check(self.lib.flash_hy_get_tuning(self.ctx, C.byref(t)))
        return t.as_dict()

    @tuning.setter
    def tuning(self, d):
        t = abi.Tuning()
        self._check(self.lib.flash_hy_get_tuning(self.ctx, C.byref(t)))
        for k, v in d.items():
            setattr(t, k, int(v))
        self._check(self.lib.flash_hy_set_tuning(self.ctx, C.byref(t)))

    def tuning_candidates(self):
        arrs = [(C.c_int * abi.TUNE_MAX)() for _ in range(3)]
        ns = [C.c_int() for _ in range(3)]
        self._check(self.lib.flash_hy_tuning_candidates(self.ctx, arrs[0], C.byref(ns[0]), arrs[1], C.byref(ns[1]),
                                                        arrs[2], C.byref(ns[2])))
        keys = ("sig_threads", "dir_threads", "mx_threads")
        return {k: list(a[:n.value]) for k, a, n in zip(keys, arrs, ns)}

    def autotune(self, dt, steps=3):
        """Time every candidate launch shape on this grid's state (restored
        afterwards) and keep the fastest: threads per CTA, then on the mixed
        path blocks per CTA (where runs are offered) and the sweep order.
        Returns (best, trials) with trials a list of (shape, ms per step)."""
        cap = 32
        best = abi.Tuning()
        table = (abi.Tuning * cap)()
        ms = (C.c_float * cap)()
        n = C.c_int()
        self._check(self.lib.flash_hy_autotune(self.ctx, float(dt), int(steps), C.byref(best), table, ms, cap,
                                               C.byref(n)))
        return best.as_dict(), [(table[q].as_dict(), float(ms[q])) for q in range(min(n.value, cap))]

    # -- sharded grids ----------------------------------------------------
    def set_owned_blocks(self, blocks):
        bl = np.ascontiguousarray(blocks, dtype=np.int32)
        self._check(self.lib.flash_hy_set_owned_blocks(self.ctx, len(bl), bl.ctypes.data_as(C.POINTER(C.c_int))))

    def set_exchange(self, send, recv):
        s = np.ascontiguousarray(send, dtype=np.int32)
        r = np.ascontiguousarray(recv, dtype=np.int32)
        self._check(self.lib.flash_hy_set_exchange(self.ctx, len(s), s.ctypes.data_as(C.POINTER(C.c_int)), len(r),
                                                   r.ctypes.data_as(C.POINTER(C.c_int))))

    def pack(self, buf):
        """Enqueue the packing of the send blocks into a device buffer (a
        CUDA tensor or a device address) on the context's stream."""
        self._check(self.lib.flash_hy_pack(self.ctx, C.c_void_p(_addr(buf))))

    def unpack(self, buf):
        self._check(self.lib.flash_hy_unpack(self.ctx, C.c_void_p(_addr(buf))))

    def step_phase(self, simTime, dt, dtOld, phase):
        """A rank's step in two phases (1: owned blocks that read no ghost
        block, 2: the rest, after unpack; see flash_hy_step_phase)."""
        self._check(self.lib.flash_hy_step_phase(self.ctx, simTime, dt, dtOld, int(phase)))

    # -- exact Riemann solver: learned guess and its training data ---------
    def set_guess_weights(self, w):
        """Attach the learned star-pressure guess (FP32 master weights, the
        layout of ExactRiemann.get_weights) to the exact-solver faces."""
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self.lib.flash_hy_set_guess_weights(self.ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))

    def harvest(self, cap, keep_log2=6):
        """Keep about one face in 2**keep_log2 (where the two-rarefaction guess
        is inexact) of the following steps' face states, at most cap."""
        self._check(self.lib.flash_hy_harvest(self.ctx, int(cap), int(keep_log2)))

    def harvest_fetch(self, torch, n_max=None):
        """The harvested face states as a [7, n] float64 CUDA tensor
        (rho_L, u_L, p_L, rho_R, u_R, p_R, gamma); starts a new sample."""
        n = C.c_longlong()
        self._check(self.lib.flash_hy_harvest_fetch(self.ctx, None, 0, C.byref(n)))
        k = n.value if n_max is None else min(n.value, int(n_max))
        out = torch.empty(7 * max(k, 1), dtype=torch.float64, device=torch.device("cuda", self.device))
        torch.cuda.current_stream(out.device).synchronize()   # the library writes on its own stream
        got = C.c_longlong()
        self._check(self.lib.flash_hy_harvest_fetch(self.ctx, C.c_void_p(out.data_ptr()), k, C.byref(got)))
        return out[:7 * got.value].view(7, got.value)

    @property
    def stream(self):
        return self.lib.flash_hy_stream(self.ctx)

    @property
    def last_launch_count(self):
        return self.lib.flash_hy_last_launch_count(self.ctx)


def _flash_ids(blocks):
    """FLASH's 1-based block IDs of 0-based block indices."""
    return np.ascontiguousarray(np.asarray(blocks, dtype=np.int64) + 1, dtype=np.int32)


def _addr(buf):
    return buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)


def next_dt(dt_cfl, dt_old, tstep_change_factor=2.0, dtmin=1e-10, dtmax=1e5):
    """Driver_computeDt.F90:431-447: limit the growth and clamp."""
    dt = min(dt_cfl, dt_old * tstep_change_factor)
    return min(max(dt, dtmin), dtmax)
