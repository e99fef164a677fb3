"""Shared problem definitions for the parity tests (small, oracle-sized)."""
import numpy as np

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid


def make_case(name, **pkw):
    """Return (grid, initial UNK, params) for a named case."""
    if name == "sod2d_x":
        g = UniformGrid(2, (8, 8), (6, 2), bc="outflow")
        return g, setups.sod(g), abi.default_params(**pkw)
    if name == "sod2d_y":       # interface normal along y
        g = UniformGrid(2, (8, 8), (2, 6), bc="outflow")
        return g, setups.sod_axis(g, axis=1), abi.default_params(**pkw)
    if name == "sod2d_rot":     # 45 degree interface, block order Morton
        g = UniformGrid(2, (8, 8), (4, 4), bc="outflow", order="morton")
        return g, setups.sod(g, xangle=45.0), abi.default_params(**pkw)
    if name == "kh2d_16":
        g = UniformGrid(2, (16, 16), (3, 3), bc="periodic")
        return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    if name == "quad2d_16":
        g = UniformGrid(2, (16, 16), (3, 3), bc="outflow")
        return g, setups.four_quadrant(g), abi.default_params(**pkw)
    if name == "sod2d_reflect":
        g = UniformGrid(2, (8, 8), (4, 3), bc="reflecting")
        return g, setups.sod(g, xangle=30.0), abi.default_params(**pkw)
    if name == "kh3d":
        g = UniformGrid(3, (8, 8, 8), (2, 3, 2), bc="periodic")
        return g, setups.kelvin_helmholtz(g), abi.default_params(gamma=5.0 / 3.0, **pkw)
    if name == "sod3d_rot":
        g = UniformGrid(3, (8, 8, 8), (3, 2, 2), bc=["outflow", "outflow", "reflecting", "reflecting",
                                                      "outflow", "outflow"])
        return g, setups.sod(g, xangle=30.0, yangle=70.0), abi.default_params(**pkw)
    raise KeyError(name)


def first_dt(oracle, unk, cap=None):
    st, dt, loc = oracle.compute_dt(unk)
    return min(dt, cap) if cap else dt
