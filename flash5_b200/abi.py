"""ctypes mirror of include/flash_hy.h and the loader of the CUDA library.

The structs here are the C-ABI parameter and grid descriptors; the library
itself is ``flash5_b200/_flash_hy.so`` built from ``flash5_b200/csrc`` by
``flash5_b200.build``.  Loading fails loudly when the library is missing:
there is no CPU fallback on the product path.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_flash_hy.so")

# status bits
OK = 0
ERR_NEG_SOUNDSPEED = 1 << 0
ERR_NONPOS_DT = 1 << 1
ERR_NEWTON_NOCONV = 1 << 2
ERR_NAN = 1 << 3
ERR_TIMEOUT = 1 << 4
ERR_BAD_ARG = 1 << 5
ERR_CUDA = 1 << 6
ERR_UNSUPPORTED = 1 << 7

RS_HLLC = 4
RS_EXACT = 100
LIM_MINMOD, LIM_MC, LIM_HYBRID, LIM_VANLEER, LIM_LIMITED = 1, 2, 3, 4, 5
BC_REFLECTING, BC_OUTFLOW, BC_PERIODIC = -31, -32, -135
PREC_FP64, PREC_FP64_FMA, PREC_MIXED = 0, 1, 2
LAYOUT_VAR_FASTEST, LAYOUT_XYZ_FASTEST = 0, 1
UPDATE_NONE, UPDATE_ALL = 0, 3


class VarMap(C.Structure):
    _fields_ = [(n, C.c_int) for n in
                ("dens", "eint", "ener", "gamc", "game", "pres", "temp", "velx", "vely", "velz", "species")]


# FLASH's alphabetical +uhd / gamma-EOS UNK ordering (1-based *_VAR).
FLASH_UHD_VARS = ("dens", "eint", "ener", "gamc", "game", "pres", "shok", "temp", "velx", "vely", "velz")


MAX_SPECIES = 16
# refinement variables of flash_hy_estimate_error (FLASH_HY_REFVAR_*)
REFVAR = {"dens": 1, "pres": 2, "velx": 3, "vely": 4, "velz": 5, "eint": 6}


def flash_varmap(nsp=0):
    """1-based *_VAR indices of FLASH's UNK; species and mass scalars (nsp of
    them) follow the property variables (SPECIES_BEGIN = NPROP_VARS + 1)."""
    vm = VarMap()
    for i, n in enumerate(FLASH_UHD_VARS):
        if hasattr(vm, n) and n != "species":
            setattr(vm, n, i + 1)
    vm.species = len(FLASH_UHD_VARS) + 1 if nsp else 0
    return vm


def with_species(params, grid):
    """A copy of params carrying the grid's species / mass-scalar counts."""
    p = Params()
    C.memmove(C.byref(p), C.byref(params), C.sizeof(Params))
    p.nspecies = getattr(grid, "nspecies", 0)
    p.nmass_scalars = getattr(grid, "nmass_scalars", 0)
    return p


class Params(C.Structure):
    _fields_ = [
        ("order", C.c_int), ("riemann_solver", C.c_int), ("slope_limiter", C.c_int),
        ("char_limiting", C.c_int), ("use_flattening", C.c_int), ("use_steepening", C.c_int),
        ("use_aux_eint", C.c_int), ("use_3d_full_ctu", C.c_int), ("precision", C.c_int),
        ("learned_guess", C.c_int),
        ("limited_slope_beta", C.c_double), ("f_pres_in_mom_flux", C.c_double), ("cfl", C.c_double),
        ("eint_switch", C.c_double), ("smlrho", C.c_double), ("smallp", C.c_double),
        ("smalle", C.c_double), ("tiny", C.c_double), ("gamma", C.c_double),
        ("gas_constant", C.c_double), ("single_species_a", C.c_double),
        ("nspecies", C.c_int), ("nmass_scalars", C.c_int),
    ]


def default_params(**kw):
    """Runtime parameters with FLASH5's unsplit defaults (unsplit/Config:105-159,
    HydroMain/Config:26, Eos/EosMain/Config:49-56) except order=3 (PPM) and
    flattening on, as in the Sod, Kelvin-Helmholtz and four-quadrant workloads."""
    p = Params()
    p.order = 3
    p.riemann_solver = RS_HLLC
    p.slope_limiter = LIM_VANLEER
    p.char_limiting = 1
    p.use_flattening = 1
    p.use_steepening = 0
    p.use_aux_eint = 1
    p.use_3d_full_ctu = 1
    p.precision = PREC_FP64
    p.learned_guess = 0
    p.limited_slope_beta = 1.0
    p.f_pres_in_mom_flux = 1.0
    p.cfl = 0.8
    p.eint_switch = 0.0
    p.smlrho = 1e-10
    p.smallp = 1e-10
    p.smalle = 1e-10
    p.tiny = 1e-16
    p.gamma = 1.4
    p.gas_constant = 8.3144598e7
    p.single_species_a = 1.0
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class GridDesc(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("nxb", C.c_int), ("nyb", C.c_int), ("nzb", C.c_int),
        ("nguard", C.c_int), ("nblocks", C.c_int), ("nblk_l1", C.c_int * 3), ("max_level", C.c_int),
        ("block_coords", C.POINTER(C.c_int)), ("block_level", C.POINTER(C.c_int)),
        ("domain_lo", C.c_double * 3), ("domain_hi", C.c_double * 3), ("bc", C.c_int * 6),
    ]


class Tuning(C.Structure):
    """flash_hy_tuning: threads per CTA of the transverse-flux/CFL passes,
    the FP64 direction kernels and the mixed direction kernels, the blocks
    per CTA along the sweep of the mixed 3D direction kernels, and the sweep
    order of the mixed path (SWEEP_XYZ or SWEEP_ZYX)."""
    _fields_ = [("sig_threads", C.c_int), ("dir_threads", C.c_int), ("mx_threads", C.c_int), ("mx_runs", C.c_int),
                ("mx_sweep", C.c_int)]

    def as_dict(self):
        return {"sig_threads": self.sig_threads, "dir_threads": self.dir_threads, "mx_threads": self.mx_threads,
                "mx_runs": self.mx_runs, "mx_sweep": self.mx_sweep}


SWEEP_XYZ, SWEEP_ZYX = 1, 2    # FLASH's constants.h values


TUNE_MAX = 8


def _set_sigs(lib):
    P, G, V = C.POINTER(Params), C.POINTER(GridDesc), C.POINTER(VarMap)
    dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
    sigs = {
        "flash_hy_create": (C.c_int, [P, G, C.c_int, C.POINTER(vp)]),
        "flash_hy_destroy": (C.c_int, [vp]),
        "flash_hy_release_memory": (C.c_int, [C.c_int]),
        "flash_hy_upload": (C.c_int, [vp, dp, C.c_int, C.c_int, V]),
        "flash_hy_download": (C.c_int, [vp, dp, C.c_int, C.c_int, V]),
        "flash_hy_step": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_int]),
        "flash_hy_step_blocks": (C.c_int, [vp, C.c_int, ip, C.c_double, C.c_double, C.c_double, C.c_int]),
        "flash_hy_compute_dt": (C.c_int, [vp, dp, ip]),
        "flash_hy_set_mesh_me": (C.c_int, [vp, C.c_int]),
        "flash_hy_dt_block": (C.c_int, [vp, ip]),
        "flash_hy_sync": (C.c_int, [vp]),
        "flash_hy_stream": (vp, [vp]),
        "flash_hy_export_state": (C.c_int, [vp, vp]),
        "flash_hy_last_error": (C.c_int, [vp, C.c_char_p, C.c_int]),
        "flash_hy_last_launch_count": (C.c_int, [vp]),
        "flash_hy_set_guess_weights": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "flash_hy_harvest": (C.c_int, [vp, C.c_longlong, C.c_int]),
        "flash_hy_harvest_fetch": (C.c_int, [vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "flash_hy_set_owned_blocks": (C.c_int, [vp, C.c_int, ip]),
        "flash_hy_set_exchange": (C.c_int, [vp, C.c_int, ip, C.c_int, ip]),
        "flash_hy_pack": (C.c_int, [vp, vp]),
        "flash_hy_unpack": (C.c_int, [vp, vp]),
        "flash_hy_step_phase": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_int]),
        "flash_hy_compute_fluxes": (C.c_int, [vp, C.c_int, ip, C.c_double, C.c_int]),
        "flash_hy_get_fluxes": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "flash_hy_put_fluxes": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "flash_hy_update_solution": (C.c_int, [vp, C.c_int, ip, C.c_double]),
        "flash_hy_estimate_error": (C.c_int, [vp, C.c_int, C.c_double, dp]),
        "flash_hy_regrid": (C.c_int, [vp, vp, C.c_int, ip, ip]),
        "flash_hy_refine_tree": (C.c_int, [G, vp, vp, C.c_int, C.c_int, ip, ip, ip, ip, ip, ip]),
        "flash_hy_mark_refine_tree": (C.c_int, [vp, C.c_int, ip, C.c_double, dp, dp, C.c_int, C.c_int, C.c_int, ip,
                                                ip, ip, ip, ip, ip]),
        "flash_hy_get_tuning": (C.c_int, [vp, C.POINTER(Tuning)]),
        "flash_hy_set_tuning": (C.c_int, [vp, C.POINTER(Tuning)]),
        "flash_hy_tuning_candidates": (C.c_int, [vp, ip, ip, ip, ip, ip, ip]),
        "flash_hy_autotune": (C.c_int, [vp, C.c_double, C.c_int, C.POINTER(Tuning), C.POINTER(Tuning),
                                        C.POINTER(C.c_float), C.c_int, ip]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_LIB = None


def load_library(path=LIB_PATH):
    """Load the CUDA C-ABI library; raise if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError(
                f"CUDA library {path} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
        _LIB = _set_sigs(C.CDLL(path))
    return _LIB
