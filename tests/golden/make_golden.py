"""Generate tests/golden/*.json with mpmath (50 significant digits).

1. sod_shocktube.json: post-shock pressure p4 of the shock-tube equation
   f(p4) = p1 [1 - (g-1)/(2g) (c5/c1) z / sqrt(1 + (g+1)/(2g) z)]^(2g/(g-1)) - p4,
   z = p4/p5 - 1 -- the function of Simulation/SimulationMain/Sod/
   shocktube.pro:15-33 -- solved by mpmath.findroot instead of the IDL
   secant iteration, for the Sod states and two harder ones.
2. riemann_star.json: star pressure and velocity of the exact ideal-gas
   Riemann problem, f_L(p) + f_R(p) + (u_R - u_L) = 0 with Toro's pressure
   functions (ch. 4, eqs. 4.6-4.7), solved to 50 digits by mpmath
   bisection + findroot, for a set of left/right states covering both
   shocks, both rarefactions, mixed waves, strong pressure ratios and both
   gammas 7/5 and 5/3.

Run: python tests/golden/make_golden.py
"""
import json
import os

import mpmath as mp

mp.mp.dps = 50
HERE = os.path.dirname(os.path.abspath(__file__))


def shocktube_f(p4, p1, p5, rho1, rho5, g):
    z = p4 / p5 - 1
    c1 = mp.sqrt(g * p1 / rho1)
    c5 = mp.sqrt(g * p5 / rho5)
    fact = (g - 1) / (2 * g) * (c5 / c1) * z / mp.sqrt(1 + (g + 1) / (2 * g) * z)
    return p1 * (1 - fact) ** (2 * g / (g - 1)) - p4


def sod_cases():
    out = []
    for (rl, pl, rr, pr, g) in [(1, 1, "0.125", "0.1", "1.4"), (1, 1000, 1, "0.01", "1.4"),
                                (1, 1, "0.125", "0.1", "1.6666666666666667")]:
        rl, pl, rr, pr, g = (mp.mpf(x) for x in (rl, pl, rr, pr, g))
        p4 = mp.findroot(lambda p: shocktube_f(p, pl, pr, rl, rr, g), (pr * 1.0001, pl * 0.9999), solver="anderson")
        out.append({"rhol": float(rl), "pl": float(pl), "rhor": float(rr), "pr": float(pr), "gamma": float(g),
                    "p4": mp.nstr(p4, 30)})
    return out


def fK(p, d, pk, g):
    c = mp.sqrt(g * pk / d)
    if p <= pk:
        return 2 * c / (g - 1) * ((p / pk) ** ((g - 1) / (2 * g)) - 1)
    A = 2 / ((g + 1) * d)
    B = (g - 1) / (g + 1) * pk
    return (p - pk) * mp.sqrt(A / (B + p))


def star(dl, ul, pl, dr, ur, pr, g):
    f = lambda p: fK(p, dl, pl, g) + fK(p, dr, pr, g) + (ur - ul)
    lo, hi = mp.mpf("1e-40"), max(pl, pr)
    while f(hi) < 0:
        hi *= 4
    for _ in range(400):
        mid = (lo + hi) / 2
        if f(mid) < 0:
            lo = mid
        else:
            hi = mid
    p = mp.findroot(f, (lo + hi) / 2)
    u = (ul + ur) / 2 + (fK(p, dr, pr, g) - fK(p, dl, pl, g)) / 2
    return p, u


def riemann_cases():
    states = [
        (1, 0, 1, "0.125", 0, "0.1", "1.4"),            # Sod
        (1, -2, "0.4", 1, 2, "0.4", "1.4"),              # two rarefactions
        (1, 0, 1000, 1, 0, "0.01", "1.4"),               # strong left shock
        (1, 0, "0.01", 1, 0, 100, "1.4"),                # strong right shock
        ("5.99924", "19.5975", "460.894", "5.99242", "-6.19633", "46.0950", "1.4"),  # colliding shocks
        ("1.5", 0, "1.5", "0.5323", "1.206", "0.3", "1.4"),          # four-quadrant pair
        (2, "0.5", "2.5", 1, "-0.5", "2.5", "1.6666666666666667"),   # KH shear pair (normal)
        ("0.001", 3, "1e-4", 1000, -3, 10, "1.6666666666666667"),   # density ratio 1e6
    ]
    out = []
    for s in states:
        dl, ul, pl, dr, ur, pr, g = (mp.mpf(x) for x in s)
        p, u = star(dl, ul, pl, dr, ur, pr, g)
        out.append({"dl": float(dl), "ul": float(ul), "pl": float(pl), "dr": float(dr), "ur": float(ur),
                    "pr": float(pr), "gamma": float(g), "pstar": mp.nstr(p, 30), "ustar": mp.nstr(u, 30)})
    return out


if __name__ == "__main__":
    with open(os.path.join(HERE, "sod_shocktube.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py (mpmath, 50 digits)", "cases": sod_cases()}, f, indent=1)
    with open(os.path.join(HERE, "riemann_star.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py (mpmath, 50 digits)", "cases": riemann_cases()}, f,
                  indent=1)
    print("wrote golden fixtures")
