"""Sweep order of the mixed-precision path (marked gpu).

The unsplit step computes every direction's face states and fluxes from the
same old state, so the order in which the direction kernels accumulate the
conservative update changes rounding only.  With tuning mx_sweep =
SWEEP_ZYX the mixed path runs z, y, x (2D: y, x): the last direction
gathers the earlier directions' internal-energy terms from their AUX slots
and applies FLASH's x, y, z formula.  The reordered FP64 sums differ in the
last bit, and the next step's FP32 reconstruction (differences of the
cells' FP64 values rounded to FP32) turns an occasional last-bit
difference into one FP32 rounding of a face-state increment, so after three
steps the two orders agree to 1e-9 of each variable's scale (floor 1), not
to the last bit; the time steps agree to 1e-12, and their locations are
equal except in mirror-symmetric problems, whose mirror cells tie.  Cases: uniform 2D and 3D grids (HLLC; exact solver with a
trained learned guess), a large eintSwitch so that every cell takes its
internal energy from the auxiliary equation (the AUX terms of all three
directions), runs of four blocks, species and mass scalars, an AMR
hierarchy.  The FP64 paths accept SWEEP_XYZ only.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro, HydroError, next_dt
from tests.cases import make_case
from tests.test_gpu_amr import amr_case

VARS = ("dens", "velx", "vely", "velz", "eint", "ener", "pres", "temp", "gamc", "game")


def _weights():
    from flash5_b200.riemann import ExactRiemann
    rs = ExactRiemann(0)
    try:
        rs.fit(rs.generate(7, 100_000), epochs=1, batch=4096)
        return rs.weights()
    finally:
        rs.close()


def _uniform(name, **kw):
    def make():
        return make_case(name, precision=abi.PREC_MIXED, **kw)
    return make


def _runs_kh():
    g = UniformGrid(3, (8, 8, 8), (8, 4, 4), bc="periodic")
    return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, precision=abi.PREC_MIXED)


def _amr_quad():
    return amr_case("quad2d_16", precision=abi.PREC_MIXED)


CASES = {
    "kh3d_hllc": _uniform("kh3d"),
    "kh3d_aux_eint": _uniform("kh3d", eint_switch=1e3),
    "sod3d_aux_eint": _uniform("sod3d_rot", eint_switch=1e3),
    "sod3d_exact_learned": _uniform("sod3d_rot", riemann_solver=abi.RS_EXACT, learned_guess=1),
    "sod2d_hllc": _uniform("sod2d_rot"),
    "kh2d_16_exact": _uniform("kh2d_16", riemann_solver=abi.RS_EXACT),
    "kh3d_species": _uniform("kh3d", nspecies=2, nmass_scalars=1),
    "kh3d_runs": _runs_kh,
    "amr_quad2d_16": _amr_quad,
}
TIES = {"sod2d_hllc", "sod3d_aux_eint", "sod3d_exact_learned"}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_zyx_sweep_matches_xyz_to_rounding(name):
    grid, unk, params = CASES[name]()
    w = _weights() if params.learned_guess else None
    xyz, zyx = Hydro(params, grid), Hydro(params, grid)
    try:
        assert xyz.tuning["mx_sweep"] == abi.SWEEP_XYZ
        zyx.tuning = dict(zyx.tuning, mx_sweep=abi.SWEEP_ZYX)
        assert zyx.tuning["mx_sweep"] == abi.SWEEP_ZYX
        for h in (xyz, zyx):
            if w is not None:
                h.set_guess_weights(w)
            h.upload(unk)
        dt, _ = xyz.compute_dt()
        t, dt_old = 0.0, dt
        for _ in range(3):
            xyz(t + dt, dt, dt_old)
            zyx(t + dt, dt, dt_old)
            t += dt
            d1, l1 = xyz.compute_dt()
            d2, l2 = zyx.compute_dt()
            assert abs(d1 - d2) <= 1e-12 * d1, (d1, d2, l1, l2)
            # symmetric problems (the rotated Sod) hold the same CFL time
            # step in mirror cells: a last-bit difference may pick the other
            if name not in TIES:
                assert tuple(l1) == tuple(l2), (l1, l2)
            dt_old, dt = dt, next_dt(d1, dt)
        a, b = grid.new_unk(), grid.new_unk()
        xyz.download(a)
        zyx.download(b)
        cols = [(v, VAR[v]) for v in VARS]
        cols += [(f"scalar{k}", c) for k, c in enumerate(range(grid.species.start, grid.species.stop))]
        for v, c in cols:
            x, y = grid.interior(a)[..., c], grid.interior(b)[..., c]
            lim = 1e-9 * max(float(np.abs(x).max()), 1.0)
            assert float(np.abs(x - y).max()) <= lim, (v, float(np.abs(x - y).max()))
    finally:
        xyz.close()
        zyx.close()


@pytest.mark.gpu
def test_fp64_paths_keep_xyz():
    grid, unk, params = make_case("kh3d")
    h = Hydro(params, grid)
    try:
        with pytest.raises(HydroError):
            h.tuning = dict(h.tuning, mx_sweep=abi.SWEEP_ZYX)
        with pytest.raises(HydroError):
            h.tuning = dict(h.tuning, mx_sweep=0)
        assert h.tuning["mx_sweep"] == abi.SWEEP_XYZ
    finally:
        h.close()
