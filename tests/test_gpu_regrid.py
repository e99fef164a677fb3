"""Refinement criterion and regrid on the GPU vs the oracle (marked gpu).

* flash_hy_estimate_error (gr_estimateBlkError) equals the oracle's
  estimator bit for bit for every block, leaves and parents, on uniform
  grids and AMR hierarchies (2D, 3D), for density and pressure, after a few
  FP64 steps;
* flash_hy_regrid (gr_updateRefinement's data movement) after marking with
  the device's errors gives the oracle's regridded leaves bit for bit, and
  the steps after it stay bit-identical too.
"""
import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.amr import mark_refine_derefine, regrid
from flash5_b200.hydro import Hydro, next_dt
from oracle import orc
from tests.cases import make_case
from tests.test_gpu_amr import VARS, amr_case
from flash5_b200.grid import VAR


def _case(name):
    if name in ("sod2d_rot", "kh3d"):
        return make_case(name)
    return amr_case(name)


def _pair_steps(h, o, ref, nsteps):
    st, dt, _ = o.compute_dt(ref)
    t, dt_old = 0.0, dt
    for _ in range(nsteps):
        assert o.hydro(ref, t + dt, dt, dt_old) == 0
        h(t + dt, dt, dt_old)
        t += dt
        st, dto, _ = o.compute_dt(ref)
        dt_old, dt = dt, next_dt(dto, dt)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d_rot", "kh3d", "kh2d_ring", "quad2d_16", "kh3d_ring"])
def test_estimator_matches_oracle(case):
    grid, unk, params = _case(case)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    h.upload(unk)
    _pair_steps(h, o, ref, 2)
    for var in ("dens", "pres"):
        got = h.estimate_error(var, 0.01)
        want = o.estimate_error(ref, var, 0.01)
        assert np.array_equal(got, want), (var, np.abs(got - want).max())
        assert np.all(np.isfinite(got)) and got.max() > 0
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["quad2d_16", "kh3d_ring"])
def test_regrid_matches_oracle(case):
    grid, unk, params = amr_case(case)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    h.upload(unk)
    _pair_steps(h, o, ref, 2)
    errs = [h.estimate_error("dens", 0.01), h.estimate_error("pres", 0.01)]
    # cutoffs from the errors themselves: refine the top 5 % of the leaves,
    # derefine under parents below the 70th percentile of the parents' errors
    lv = np.concatenate([e[grid.leaf_ids] for e in errs])
    pv = np.concatenate([e[~grid.is_leaf] for e in errs])
    refine, derefine = mark_refine_derefine(grid, errs, np.quantile(lv, 0.95), np.quantile(pv, 0.7))
    g2, src, how = regrid(grid, refine, derefine)
    assert np.any(how == 1) and np.any(how == 2), "the case must refine and derefine"
    h2 = h.regrid(g2, src, how)
    h.close()
    ref2 = o.regrid(ref, g2, src, how)
    out = g2.new_unk()
    h2.download(out)
    leaves = g2.leaf_ids
    a, b = g2.interior(out)[leaves], g2.interior(ref2)[leaves]
    for v in VARS:
        assert np.array_equal(a[..., VAR[v]], b[..., VAR[v]]), (v, np.abs(a[..., VAR[v]] - b[..., VAR[v]]).max())
    o2 = orc.Oracle(params, g2)
    dtg, locg = h2.compute_dt()
    st, dto, loco = o2.compute_dt(ref2)
    assert dtg == dto and tuple(locg) == tuple(loco)
    _pair_steps(h2, o2, ref2, 2)
    h2.download(out)
    h2.close()
    a, b = g2.interior(out)[leaves], g2.interior(ref2)[leaves]
    for v in VARS:
        assert np.array_equal(a[..., VAR[v]], b[..., VAR[v]]), (v, np.abs(a[..., VAR[v]] - b[..., VAR[v]]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case,rc,dc", [("kh2d_ring", 0.8, 0.2), ("quad2d_16", 0.3, 0.6), ("kh3d_ring", 0.5, 0.4),
                                        ("sod2d_reflect", 0.05, 0.9)])
def test_device_marks_and_tree_equal_the_host_path(case, rc, dc):
    """flash_hy_mark_refine_tree (estimator, FLASH's marks and PARAMESH's
    tree rules as kernels) returns the tree of the host path -- device
    estimator, amr.mark_refine_derefine, flash_hy_refine_tree -- node for
    node: levels, coordinates, parents, and the regrid's src / how; the
    cutoffs are chosen so that refinement, 2:1 balance and derefinement all
    occur."""
    from flash5_b200.amr import regrid_native
    grid, unk, params = _case(case)
    h = Hydro(params, grid)
    try:
        h.upload(unk)
        dt, _ = h.compute_dt()
        for _ in range(2):
            h(dt, dt, dt)
        errs = [h.estimate_error(v, 0.01) for v in ("dens", "pres")]
        r, d = mark_refine_derefine(grid, errs, rc, dc)
        g2, src, how = regrid_native(grid, r, d)
        lev, coords, par, src_d, how_d = h.mark_refine_tree(("dens", "pres"), 0.01, rc, dc)
    finally:
        h.close()
    assert np.array_equal(lev, g2.levels)
    assert np.array_equal(coords, g2.coords)
    assert np.array_equal(par, g2.parent)
    assert np.array_equal(src_d, src) and np.array_equal(how_d, how)
    assert r.any() or d.any()
