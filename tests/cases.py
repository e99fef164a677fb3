"""Shared problem definitions for the parity tests (small, oracle-sized)."""
import numpy as np

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid


def make_case(name, nspecies=0, nmass_scalars=0, **pkw):
    """Return (grid, initial UNK, params) for a named case, with nspecies
    species and nmass_scalars mass scalars (setups.add_species)."""
    grid, unk, params = _make_case(name, {"nspecies": nspecies, "nmass_scalars": nmass_scalars}, **pkw)
    setups.add_species(grid, unk)
    return grid, unk, params


def _make_case(name, sk, **pkw):
    if name == "sod2d_x":
        g = UniformGrid(2, (8, 8), (6, 2), bc="outflow", **sk)
        return g, setups.sod(g), abi.default_params(**pkw)
    if name == "sod2d_y":       # interface normal along y
        g = UniformGrid(2, (8, 8), (2, 6), bc="outflow", **sk)
        return g, setups.sod_axis(g, axis=1), abi.default_params(**pkw)
    if name == "sod2d_rot":     # 45 degree interface, block order Morton
        g = UniformGrid(2, (8, 8), (4, 4), bc="outflow", order="morton", **sk)
        return g, setups.sod(g, xangle=45.0), abi.default_params(**pkw)
    if name == "kh2d_16":
        g = UniformGrid(2, (16, 16), (3, 3), bc="periodic", **sk)
        return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    if name == "quad2d_16":
        g = UniformGrid(2, (16, 16), (3, 3), bc="outflow", **sk)
        return g, setups.four_quadrant(g), abi.default_params(**pkw)
    if name == "sod2d_reflect":
        g = UniformGrid(2, (8, 8), (4, 3), bc="reflecting", **sk)
        return g, setups.sod(g, xangle=30.0), abi.default_params(**pkw)
    if name == "kh3d":
        g = UniformGrid(3, (8, 8, 8), (2, 3, 2), bc="periodic", **sk)
        return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    if name == "sod3d_rot":
        g = UniformGrid(3, (8, 8, 8), (3, 2, 2), bc=["outflow", "outflow", "reflecting", "reflecting",
                                                      "outflow", "outflow"], **sk)
        return g, setups.sod(g, xangle=30.0, yangle=70.0), abi.default_params(**pkw)
    raise KeyError(name)


def first_dt(oracle, unk, cap=None):
    st, dt, loc = oracle.compute_dt(unk)
    return min(dt, cap) if cap else dt
