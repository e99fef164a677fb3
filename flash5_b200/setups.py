"""Initial conditions of the benchmark problems, written into FLASH UNK arrays.

* ``sod``: Simulation/SimulationMain/Sod/Simulation_initBlock.F90:139-290
  (left/right states, the averaged interface cell and the rotated interface
  of Simulation_init.F90:107-125).
* ``kelvin_helmholtz``: the 3D shear layer of the benchmark description
  (rho=2, vx=+0.5 for |y-0.5|<0.25, rho=1, vx=-0.5 elsewhere, p=2.5,
  vy = 0.01 sin(4 pi x) + seeded uniform noise of amplitude 1e-3).  FLASH5
  ships no KH setup; the noise comes from numpy's PCG64 seeded with 12345
  and is drawn in global (z, y, x) cell order so it does not depend on the
  block decomposition.
* ``four_quadrant``: the 2D four-state Riemann problem of the benchmark
  description (Lax-Liu configuration 3 states; quadrant 1 is x>0.5, y>0.5,
  counted counter-clockwise).

Every setup fills DENS, VEL*, PRES, EINT, ENER (= max(eint + ekin, smallp)
as in the Sod initBlock), GAMC = GAME = gamma and TEMP = 1e-10; the caller
then applies the EOS in MODE_DENS_EI, as Grid_initDomain does.
"""
import numpy as np

from .grid import VAR


def _fill(grid, unk, rho, vx, vy, vz, p, gamma, smallp=1e-10):
    it = grid.interior(unk)
    ekin = 0.5 * (vx ** 2 + vy ** 2 + vz ** 2)
    eint = p / (gamma - 1.0)
    eint = eint / rho
    ener = np.maximum(eint + ekin, smallp)
    it[..., VAR["dens"]] = rho
    it[..., VAR["pres"]] = p
    it[..., VAR["velx"]] = vx
    it[..., VAR["vely"]] = vy
    it[..., VAR["velz"]] = vz
    it[..., VAR["ener"]] = ener
    it[..., VAR["eint"]] = eint
    it[..., VAR["game"]] = gamma
    it[..., VAR["gamc"]] = gamma
    it[..., VAR["temp"]] = 1.0e-10
    return unk


def sod(grid, gamma=1.4, rho_l=1.0, rho_r=0.125, p_l=1.0, p_r=0.1, u_l=0.0, u_r=0.0,
        posn=0.5, xangle=0.0, yangle=90.0):
    """Sod shock tube (Simulation_initBlock.F90:139-290)."""
    unk = grid.new_unk()
    xa = xangle * 0.0174532925
    ya = yangle * 0.0174532925
    xcos = np.cos(xa)
    if grid.ndim == 2:
        ycos = np.sqrt(1.0 - xcos * xcos)
        zcos = 0.0
    else:
        ycos = np.cos(ya)
        zcos = np.sqrt(max(0.0, 1.0 - xcos * xcos - ycos * ycos))
    x, y, z = grid.cell_centers()
    xl, xr = grid.cell_edges(0)
    lposn = posn - z * zcos / xcos - y * ycos / xcos
    left = xr <= lposn
    mid = (xl < lposn) & (xr > lposn)
    rho = np.where(left, rho_l, np.where(mid, 0.5 * (rho_l + rho_r), rho_r))
    p = np.where(left, p_l, np.where(mid, 0.5 * (p_l + p_r), p_r))
    u = np.where(left, u_l, np.where(mid, 0.5 * (u_l + u_r), u_r))
    return _fill(grid, unk, rho, u * xcos, u * ycos, u * zcos, p, gamma)


def sod_axis(grid, axis=0, gamma=1.4, rho_l=1.0, rho_r=0.125, p_l=1.0, p_r=0.1, posn=0.5):
    """Planar Sod problem with its interface normal along ``axis`` (the
    angled form of ``sod`` divides by cos(xangle) and cannot express an
    interface normal to y or z)."""
    unk = grid.new_unk()
    c = grid.cell_centers()[axis]
    left = c < posn
    rho = np.where(left, rho_l, rho_r)
    p = np.where(left, p_l, p_r)
    z = np.zeros_like(rho)
    return _fill(grid, unk, rho, z, z, z, p, gamma)


def _block_noise(grid, seed, amp):
    """Seeded uniform noise drawn in global (z, y, x) cell order on the
    finest level, so it does not depend on the block decomposition; a block
    of a coarser AMR level gets the average over its footprint."""
    L = getattr(grid, "max_used_level", 1)
    f = 2 ** (L - 1)
    nx, ny, nz = (grid.nblk[d] * grid.nb[d] * (f if d < grid.ndim else 1) for d in range(3))
    rng = np.random.default_rng(seed)
    glob = rng.uniform(-amp, amp, size=(nz, ny, nx))
    out = np.empty((grid.nblocks, grid.nb[2], grid.nb[1], grid.nb[0]))
    levels = getattr(grid, "levels", np.ones(grid.nblocks, dtype=np.int32))
    for b in range(grid.nblocks):
        r = 2 ** (L - levels[b])
        o = [grid.coords[b, d] * grid.nb[d] * r if d < grid.ndim else 0 for d in range(3)]
        e = [grid.nb[d] * r if d < grid.ndim else 1 for d in range(3)]
        t = glob[o[2]:o[2] + e[2], o[1]:o[1] + e[1], o[0]:o[0] + e[0]]
        if r > 1:
            rz = r if grid.ndim > 2 else 1
            t = t.reshape(grid.nb[2], rz, grid.nb[1], r, grid.nb[0], r).mean(axis=(1, 3, 5))
        out[b] = t
    return out


def kelvin_helmholtz(grid, gamma=5.0 / 3.0, seed=12345, noise=1e-3):
    """3D (or 2D) Kelvin-Helmholtz shear layer with seeded noise."""
    unk = grid.new_unk()
    x, y, z = grid.cell_centers()
    inner = np.abs(y - 0.5) < 0.25
    rho = np.where(inner, 2.0, 1.0)
    vx = np.where(inner, 0.5, -0.5)
    pert = _block_noise(grid, seed, noise)
    vy = 0.01 * np.sin(4.0 * np.pi * x) + pert
    vz = np.zeros_like(rho)
    p = np.full_like(rho, 2.5)
    return _fill(grid, unk, rho, vx, vy, vz, p, gamma)


QUADRANTS = {  # (rho, u, v, p)
    1: (1.5, 0.0, 0.0, 1.5),
    2: (0.5323, 1.206, 0.0, 0.3),
    3: (0.138, 1.206, 1.206, 0.029),
    4: (0.5323, 0.0, 1.206, 0.3),
}


def four_quadrant(grid, gamma=1.4, x0=0.5, y0=0.5):
    unk = grid.new_unk()
    x, y, z = grid.cell_centers()
    q = np.where(x > x0, np.where(y > y0, 1, 4), np.where(y > y0, 2, 3))
    vals = np.zeros(q.shape + (4,))
    for k, s in QUADRANTS.items():
        vals[q == k] = s
    return _fill(grid, unk, vals[..., 0], vals[..., 1], vals[..., 2], np.zeros_like(vals[..., 0]),
                 vals[..., 3], gamma)


def uniform(grid, rho=1.0, v=(0.0, 0.0, 0.0), p=1.0, gamma=1.4):
    unk = grid.new_unk()
    shape = (grid.nblocks, grid.nb[2], grid.nb[1], grid.nb[0])
    f = lambda a: np.full(shape, a, dtype=np.float64)
    return _fill(grid, unk, f(rho), f(v[0]), f(v[1]), f(v[2]), f(p), gamma)


def add_species(grid, unk, width=0.05):
    """Fill the species and mass scalars of a grid's UNK (grid.nspecies,
    grid.nmass_scalars): species 0 is 1 inside the band |y - 0.5| < 0.25
    (smoothed over `width`, the dense layer of the Kelvin-Helmholtz setup),
    further species share the rest in fixed proportions so that the species
    sum to 1; mass scalar m is a smooth passive tracer
    0.5 + 0.4 sin(2 pi (m + 1) x) cos(2 pi y).  Synthetic: FLASH5's
    Simulation units define their own species."""
    ns, nm = grid.nspecies, grid.nmass_scalars
    if ns + nm == 0:
        return unk
    it = grid.interior(unk)
    x, y, z = grid.cell_centers()
    band = 0.5 * (np.tanh((0.25 - np.abs(y - 0.5)) / width) + 1.0)
    base = grid.species.start
    if ns:
        it[..., base] = band if ns > 1 else 1.0
        rest = 1.0 - band
        w = np.arange(1, ns, dtype=np.float64)
        w = w / w.sum() if ns > 1 else w
        for s in range(1, ns):
            it[..., base + s] = rest * w[s - 1]
    for m in range(nm):
        it[..., base + ns + m] = 0.5 + 0.4 * np.sin(2 * np.pi * (m + 1) * x) * np.cos(2 * np.pi * y)
    return unk
