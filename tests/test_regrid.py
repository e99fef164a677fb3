"""Refinement marking, the regridded tree and the oracle's regrid (CPU).

* mark_refine_derefine follows gr_markRefineDerefine.F90: refinement above
  the refine cutoff (not beyond max_refine), derefinement of leaves whose
  error and whose parent's error are at or below the derefine cutoff,
  leaves only;
* the regridded tree is a proper PARAMESH tree (complete sibling sets,
  neighbours -- diagonals included -- within one level) and its map to the
  old tree is consistent; refining every leaf and derefining them again
  gives the original tree back;
* the oracle's regrid keeps a uniform state uniform and prolongs a linear
  field exactly away from the boundaries.
"""
import itertools

import numpy as np

from flash5_b200 import abi, setups
from flash5_b200.amr import AmrGrid, indicator_refiner, mark_refine_derefine, regrid
from flash5_b200.grid import VAR
from oracle import orc


def ring(max_level=3, bc="periodic"):
    g = AmrGrid(2, (8, 8), (4, 4), max_level, bc=bc)
    f = lambda X, Y, Z: 1.0 + 0.8 * np.tanh(((X - 0.5) ** 2 + (Y - 0.45) ** 2 - 0.04) / 0.004)
    g.refine_levels(indicator_refiner(g, f, 0.05))
    return g


def balanced(g):
    leaves = {(int(g.levels[b]), tuple(int(v) for v in g.coords[b])) for b in g.leaf_ids}
    cover = {}
    for lev, c in leaves:
        cover[(lev, c)] = lev
    # every leaf's neighbours (diagonals included) are leaves within one level
    offs = [o for o in itertools.product((-1, 0, 1), repeat=g.ndim) if any(o)]
    for lev, c in leaves:
        for o in offs:
            o3 = tuple(o) + (0,) * (3 - g.ndim)
            found = False
            for dl in (-1, 0, 1):
                L = lev + dl
                if L < 1 or L > g.max_level:
                    continue
                # the position of the neighbour cell centre on level L
                p = []
                ok = True
                for d in range(3):
                    if d >= g.ndim:
                        p.append(0)
                        continue
                    # neighbour block of (lev, c) offset o, mapped to level L
                    x = (c[d] + o3[d]) * 2 ** max(dl, 0) if dl >= 0 else (c[d] + o3[d]) // 2
                    ext = g.nblk[d] * 2 ** (L - 1)
                    if x < 0 or x >= ext:
                        if not g.periodic[d]:
                            ok = False
                            break
                        x %= ext
                    p.append(x)
                if not ok:
                    found = True
                    break
                if (L, tuple(p)) in leaves or (dl == 1 and any((L, tuple(q)) in leaves for q in [tuple(p)])):
                    found = True
                    break
                if dl == 1:
                    # a finer neighbour: some child touching the block is a leaf
                    for ch in itertools.product((0, 1), repeat=g.ndim):
                        q = tuple(p[d] + (ch[d] if d < g.ndim else 0) for d in range(3))
                        if (L, q) in leaves:
                            found = True
                    if found:
                        break
            if not found:
                return False
    return True


def test_marking_rules():
    g = ring()
    n = g.nblocks
    err = np.zeros(n)
    leaves = g.leaf_ids
    err[leaves[0]] = 0.9
    err[leaves[1]] = 0.5
    refine, derefine = mark_refine_derefine(g, [err], 0.8, 0.2)
    assert refine[leaves[0]] == (g.levels[leaves[0]] < g.max_level)
    assert not derefine[leaves[0]] and not derefine[leaves[1]] and not refine[leaves[1]]
    assert np.all(derefine[leaves[2:]] | (err[np.maximum(g.parent[leaves[2:]], 0)] > 0.2)
                  | (g.parent[leaves[2:]] < 0) | derefine[leaves[2:]])
    assert not np.any(refine[~g.is_leaf]) and not np.any(derefine[~g.is_leaf])
    # a parent above the derefine cutoff keeps its children
    p = g.parent[leaves[-1]]
    err2 = np.zeros(n)
    err2[p] = 0.3
    _, der2 = mark_refine_derefine(g, [err2], 0.8, 0.2)
    kids = np.nonzero(g.parent == p)[0]
    assert not np.any(der2[kids])


def test_regrid_tree_and_round_trip():
    g = ring()
    n = g.nblocks
    rng = np.random.default_rng(3)
    refine = g.is_leaf & (rng.random(n) < 0.3)
    derefine = g.is_leaf & ~refine & (rng.random(n) < 0.6)
    g2, src, how = regrid(g, refine, derefine)
    assert balanced(g2)
    for q in range(g2.nblocks):
        o = src[q]
        if how[q] == 0:
            assert g2.levels[q] == g.levels[o] and np.array_equal(g2.coords[q], g.coords[o])
        elif how[q] == 1:
            assert g.is_leaf[o] and g2.levels[q] == g.levels[o] + 1
            assert np.array_equal(g2.coords[q][:2] // 2, g.coords[o][:2])
        else:
            assert not g.is_leaf[o] and g2.is_leaf[q]
    # refine every leaf below max_level, then derefine the new leaves again
    g3, _, _ = regrid(g, g.is_leaf.copy(), np.zeros(n, dtype=bool))
    assert balanced(g3)
    new = np.zeros(g3.nblocks, dtype=bool)
    old_keys = {(int(g.levels[b]), tuple(g.coords[b])) for b in range(n)}
    for b in g3.leaf_ids:
        new[b] = (int(g3.levels[b]), tuple(g3.coords[b])) not in old_keys
    g4, _, _ = regrid(g3, np.zeros(g3.nblocks, dtype=bool), new)
    k = lambda gg: sorted((int(gg.levels[b]), tuple(gg.coords[b]), bool(gg.is_leaf[b])) for b in range(gg.nblocks))
    assert k(g4) == k(g)


def test_oracle_regrid_uniform_and_linear():
    g = ring(bc="outflow")
    params = abi.default_params()
    u = setups.uniform(g, rho=1.3, v=(0.2, -0.1, 0.0), p=0.7)
    o = orc.Oracle(params, g)
    o.eos_init(u)
    refine = g.is_leaf & (g.levels < g.max_level)
    g2, src, how = regrid(g, refine, np.zeros(g.nblocks, dtype=bool))
    out = o.regrid(u.copy(), g2, src, how)
    it = g2.interior(out)[g2.leaf_ids]
    assert np.allclose(it[..., VAR["dens"]], 1.3, rtol=1e-14, atol=0)
    assert np.allclose(it[..., VAR["velx"]], 0.2, rtol=1e-14, atol=0)
    assert np.allclose(it[..., VAR["pres"]], 0.7, rtol=1e-13, atol=0)
    # a linear density: new children away from the domain boundary exact
    x, y, z = g.cell_centers()
    u2 = setups.uniform(g, rho=1.0, p=1.0)
    g.interior(u2)[..., VAR["dens"]] = 1.0 + 0.25 * x + 0.125 * y
    o.eos_init(u2)
    out2 = o.regrid(u2.copy(), g2, src, how)
    x2, y2, _ = g2.cell_centers()
    kids = np.nonzero((how == 1) & g2.is_leaf)[0]
    inner = [q for q in kids if np.all(g2.coords[q][:2] > 0) and
             np.all(g2.coords[q][:2] < np.array(g2._extent(int(g2.levels[q]))[:2]) - 1)]
    assert inner
    d = g2.interior(out2)[inner][..., VAR["dens"]]
    exact = 1.0 + 0.25 * x2[inner] + 0.125 * y2[inner]
    assert np.abs(d - exact).max() < 1e-13


def _same_grid(a, b):
    assert a.nblocks == b.nblocks
    assert np.array_equal(a.levels, b.levels) and np.array_equal(a.coords, b.coords)
    assert np.array_equal(a.parent, b.parent) and np.array_equal(a.is_leaf, b.is_leaf)
    assert np.array_equal(a.delta_b, b.delta_b)


def test_native_tree_matches_python():
    from flash5_b200.amr import regrid_native
    cases = [ring(), ring(bc="outflow"),
             AmrGrid(3, (8, 8, 8), (2, 2, 2), 3, bc="periodic")]
    f3 = lambda X, Y, Z: 1.0 + 0.8 * np.tanh(((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.5) ** 2 - 0.06) / 0.004)
    cases[2].refine_levels(indicator_refiner(cases[2], f3, 0.05))
    rng = np.random.default_rng(7)
    for g in cases:
        for trial in range(3):
            n = g.nblocks
            refine = g.is_leaf & (rng.random(n) < 0.2)
            derefine = g.is_leaf & ~refine & (rng.random(n) < 0.7)
            a, sa, ha = regrid(g, refine, derefine)
            b, sb, hb = regrid_native(g, refine, derefine)
            _same_grid(a, b)
            assert np.array_equal(sa, sb) and np.array_equal(ha, hb)
