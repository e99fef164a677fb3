"""Cell-by-cell comparison metrics -- TEST INFRASTRUCTURE ONLY.

Restates the comparison of the reference's tools/sfocu/sfocu.c: the
relative difference of one cell (line 32), the L1 relative norm
sum|a-b| / sum|b| accumulated cell by cell (lines 814-846) and the
magnitude error max|a-b| / max|b| (lines 870-875).
"""
import numpy as np


def l1_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def mag_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())


CONSERVED = ("dens", "xmom", "ymom", "zmom", "ener")


def conserved(unk_interior, var):
    """(rho, rho u, rho v, rho w, rho E) from UNK interiors (VAR index map)."""
    r = unk_interior[..., var["dens"]]
    return {
        "dens": r,
        "xmom": r * unk_interior[..., var["velx"]],
        "ymom": r * unk_interior[..., var["vely"]],
        "zmom": r * unk_interior[..., var["velz"]],
        "ener": r * unk_interior[..., var["ener"]],
    }


def compare(unk_a, unk_b, grid):
    """Per conserved variable {name: (L1 rel, mag err)} over block interiors."""
    from flash5_b200.grid import VAR
    ca = conserved(grid.interior(unk_a), VAR)
    cb = conserved(grid.interior(unk_b), VAR)
    return {k: (l1_rel(ca[k], cb[k]), mag_err(ca[k], cb[k])) for k in CONSERVED}
