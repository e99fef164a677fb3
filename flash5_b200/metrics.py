"""Error norms of the benchmark reports: the comparison of FLASH's
tools/sfocu/sfocu.c, per conserved variable -- the L1 relative norm
sum|a-b| / sum|b| accumulated cell by cell (lines 814-846) and the
magnitude error max|a-b| / max|b| (lines 870-875)."""
import numpy as np

CONSERVED = ("dens", "xmom", "ymom", "zmom", "ener")


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


def conserved(unk, var):
    """(rho, rho u, rho v, rho w, rho E) of UNK cells (VAR index map)."""
    r = unk[..., var["dens"]]
    return {"dens": r, "xmom": r * unk[..., var["velx"]], "ymom": r * unk[..., var["vely"]],
            "zmom": r * unk[..., var["velz"]], "ener": r * unk[..., var["ener"]]}


def conserved_l1(a, b, var):
    """{conserved variable: L1 relative norm of a against b}."""
    ca, cb = conserved(a, var), conserved(b, var)
    return {k: l1_rel(ca[k], cb[k]) for k in CONSERVED}


def conserved_linf(a, b, var):
    """{conserved variable: magnitude error max|a-b| / max|b| of a against b}."""
    ca, cb = conserved(a, var), conserved(b, var)
    return {k: mag_err(ca[k], cb[k]) for k in CONSERVED}
