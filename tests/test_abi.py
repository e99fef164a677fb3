"""C-ABI library: loads without a GPU and exports every declared symbol;
host-side parameter/grid marshalling matches the header."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.grid import UniformGrid
from flash5_b200.hydro import next_dt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(flash_hy_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("flash_hy_create", "flash_hy_destroy", "flash_hy_upload", "flash_hy_download", "flash_hy_step",
              "flash_hy_step_blocks", "flash_hy_compute_dt", "flash_hy_last_error"):
        assert n in names


def test_library_loads_and_exports_every_declared_symbol():
    lib = abi.load_library()
    for n in declared_functions():
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(flash_hy_\w+)\b", out))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_header():
    # offsets computed by the C compiler from include/flash_hy.h
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "flash_hy.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(flash_hy_params), offsetof(flash_hy_params, limited_slope_beta),
         offsetof(flash_hy_params, single_species_a), sizeof(flash_hy_grid_desc),
         offsetof(flash_hy_grid_desc, block_coords), offsetof(flash_hy_grid_desc, bc));
  printf("%zu\n", sizeof(flash_hy_varmap));
  printf("%zu %zu\n", sizeof(flash_hy_tuning), offsetof(flash_hy_tuning, mx_sweep));
  return 0;
}'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    assert vals[0] == C.sizeof(abi.Params)
    assert vals[1] == abi.Params.limited_slope_beta.offset
    assert vals[2] == abi.Params.single_species_a.offset
    assert vals[3] == C.sizeof(abi.GridDesc)
    assert vals[4] == abi.GridDesc.block_coords.offset
    assert vals[5] == abi.GridDesc.bc.offset
    assert vals[6] == C.sizeof(abi.VarMap)
    assert vals[7] == C.sizeof(abi.Tuning)
    assert vals[8] == abi.Tuning.mx_sweep.offset


def test_flash_varmap_is_alphabetical():
    vm = abi.flash_varmap()
    assert (vm.dens, vm.eint, vm.ener, vm.gamc, vm.game, vm.pres, vm.temp, vm.velx, vm.vely, vm.velz) == \
        (1, 2, 3, 4, 5, 6, 8, 9, 10, 11)


def test_create_rejects_bad_arguments_without_touching_the_gpu():
    lib = abi.load_library()
    g = UniformGrid(2, (8, 8), (2, 2))
    gd = g.desc()
    ctx = C.c_void_p()
    p = abi.default_params(order=2)
    assert lib.flash_hy_create(C.byref(p), C.byref(gd), 0, C.byref(ctx)) == abi.ERR_UNSUPPORTED
    p = abi.default_params(gamma=1.0)
    assert lib.flash_hy_create(C.byref(p), C.byref(gd), 0, C.byref(ctx)) == abi.ERR_BAD_ARG
    g = UniformGrid(2, (12, 12), (2, 2))
    gd = g.desc()
    assert lib.flash_hy_create(C.byref(abi.default_params()), C.byref(gd), 0, C.byref(ctx)) == abi.ERR_UNSUPPORTED
    assert lib.flash_hy_step(None, 0.0, 1.0, 1.0, 0) == abi.ERR_BAD_ARG
    # the learned guess belongs to the exact solver on the mixed path
    g = UniformGrid(2, (8, 8), (2, 2))
    gd = g.desc()
    for kw in (dict(learned_guess=1), dict(learned_guess=1, riemann_solver=abi.RS_EXACT),
               dict(learned_guess=1, precision=abi.PREC_MIXED), dict(riemann_solver=1)):
        p = abi.default_params(**kw)
        assert lib.flash_hy_create(C.byref(p), C.byref(gd), 0, C.byref(ctx)) == abi.ERR_UNSUPPORTED, kw
    assert lib.flash_hy_set_guess_weights(None, None, 0) == abi.ERR_BAD_ARG
    assert lib.flash_hy_harvest(None, 10, 0) == abi.ERR_BAD_ARG
    # nothing cached yet: releasing the kept device memory touches no device
    assert lib.flash_hy_release_memory(-1) == 0


def test_grid_descriptor_and_unk_layout():
    g = UniformGrid(3, (8, 8, 8), (2, 3, 4), bc="periodic", order="morton")
    d = g.desc()
    assert d.nblocks == 24 and tuple(d.nblk_l1) == (2, 3, 4)
    coords = np.ctypeslib.as_array(d.block_coords, shape=(72,)).reshape(24, 3)
    assert len({tuple(c) for c in coords}) == 24
    assert g.new_unk().shape == (24, 16, 16, 16, 11)
    assert g.delta == (0.5 / 8, 1 / 24, 1 / 32)


def test_driver_dt_policy():
    assert next_dt(1.0, 0.1) == 0.2           # growth limited to tstepChangeFactor = 2
    assert next_dt(0.05, 0.1) == 0.05
    assert next_dt(1e-20, 1.0) == 1e-10       # dtmin clamp
