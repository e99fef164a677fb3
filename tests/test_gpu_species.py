"""Species and mass scalars on the GPU (marked gpu), through the C ABI.

* FP64: the species, mass scalars and every hydro variable equal the
  oracle bit for bit after several steps (2D and 3D with the full CTU;
  periodic, outflow and reflecting boundaries), and so does a FLASH4-style
  block-list step;
* the hydro variables are bit-identical with and without species;
* mixed precision: species within 1e-6 relative L1 of the FP64 GPU run;
* species on AMR hierarchies (restriction, guard cells, the species flux
  register) and through a regrid equal the oracle bit for bit (FP64), and
  stay within 1e-6 relative L1 of it on the mixed path;
* the split step keeps the species fluxes after the hydro fluxes in FLASH's
  flux arrays (equal to the oracle's) and, with or without a get/put round
  trip, updates as the fused step does; a replaced mass-scalar flux changes
  exactly the two cells beside the face.
"""
import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.grid import NUNK, VAR
from flash5_b200.hydro import Hydro, next_dt
from oracle import orc
from tests.cases import make_case


def _steps(h, o, unk, ref, steps, blocks=None):
    h.upload(unk)
    dt, _ = h.compute_dt()
    t, dt_old = 0.0, dt
    for _ in range(steps):
        if blocks is None:
            h(t + dt, dt, dt_old)
        else:
            h.step_blocks(blocks, t + dt, dt, dt_old)
        if o is not None:
            assert o.hydro(ref, t + dt, dt, dt_old, blocks=blocks) == 0
        t += dt
        dts, _ = h.compute_dt()
        dt_old, dt = dt, next_dt(dts, dt)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_16", "sod2d_reflect", "kh3d", "sod3d_rot"])
def test_fp64_species_match_oracle(case):
    grid, unk, params = make_case(case, nspecies=2, nmass_scalars=1)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    _steps(h, o, unk, ref, 4)
    out = grid.new_unk()
    h.download(out)
    h.close()
    a, b = grid.interior(out), grid.interior(ref)
    sp = grid.species
    assert np.array_equal(a[..., sp], b[..., sp]), np.abs(a[..., sp] - b[..., sp]).max()
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_block_list_step_with_species_matches_oracle():
    grid, unk, params = make_case("kh3d", nspecies=1, nmass_scalars=2)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    blocks = list(range(grid.nblocks))[1::2]
    _steps(h, o, unk, ref, 2, blocks=blocks)
    out = grid.new_unk()
    h.download(out)
    h.close()
    assert np.array_equal(grid.interior(out), grid.interior(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_hydro_unchanged_by_species(prec):
    g0, u0, p0 = make_case("kh3d", precision=prec)
    g1, u1, p1 = make_case("kh3d", nspecies=2, nmass_scalars=1, precision=prec)
    outs = []
    for g, u, p in ((g0, u0, p0), (g1, u1, p1)):
        h = Hydro(p, g)
        _steps(h, None, u, None, 3)
        out = g.new_unk()
        h.download(out)
        h.close()
        outs.append(g.interior(out))
    assert np.array_equal(outs[0], outs[1][..., :NUNK])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh3d", "kh2d_16"])
def test_mixed_species_within_tolerance(case):
    runs = []
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        grid, unk, params = make_case(case, nspecies=2, nmass_scalars=1, precision=prec)
        h = Hydro(params, grid)
        _steps(h, None, unk, None, 4)
        out = grid.new_unk()
        h.download(out)
        h.close()
        runs.append(grid.interior(out)[..., grid.species])
    a, b = runs
    l1 = np.abs(b - a).sum(axis=(0, 1, 2, 3)) / np.abs(a).sum(axis=(0, 1, 2, 3))
    assert np.all(l1 <= 1e-6), l1
    assert np.abs(b[..., 0] + b[..., 1] - 1.0).max() < 1e-14


def _state(h, grid):
    out = grid.new_unk()
    h.download(out)
    return grid.interior(out).copy()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d_rot", "kh3d"])
def test_split_step_species_fluxes_match_oracle(case):
    """compute_fluxes keeps the species fluxes F_dens * X after the 8 hydro
    fluxes (NFLUXES = 8 + species + mass scalars), equal to the oracle's."""
    grid, unk, params = make_case(case, nspecies=2, nmass_scalars=1)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    h.upload(unk)
    dt, _ = h.compute_dt()
    blocks = [0, grid.nblocks // 2, grid.nblocks - 1]
    h.compute_fluxes(blocks, dt, abi.UPDATE_NONE)
    for b in blocks:
        st, want = o.block_fluxes(ref.copy(), b, dt)
        assert want.shape[-1] == 11
        for d in range(grid.ndim):
            got = h.get_fluxes(b, d + 1)
            assert np.array_equal(got, want[d]), (b, d, np.abs(got - want[d]).max(axis=0))
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case,prec", [("sod2d_rot", abi.PREC_FP64), ("kh3d", abi.PREC_FP64),
                                       ("kh3d", abi.PREC_MIXED)])
def test_split_step_with_species_equals_fused_step(case, prec):
    grid, unk, params = make_case(case, nspecies=2, nmass_scalars=1, precision=prec)
    blocks = list(range(grid.nblocks))[1::2]
    fused, split, both = Hydro(params, grid), Hydro(params, grid), Hydro(params, grid)
    for h in (fused, split, both):
        h.upload(unk)
    dt, _ = fused.compute_dt()
    before = _state(split, grid)
    fused.step_blocks(blocks, dt, dt, dt)
    split.compute_fluxes(blocks, dt, abi.UPDATE_NONE)
    assert np.array_equal(_state(split, grid), before)
    for blk in blocks[:2]:                                      # a get/put round trip changes nothing
        for d in range(1, grid.ndim + 1):
            split.put_fluxes(blk, d, split.get_fluxes(blk, d))
    split.update_solution(blocks, dt)
    both.compute_fluxes(blocks, dt, abi.UPDATE_ALL)
    a, b, c = _state(fused, grid), _state(split, grid), _state(both, grid)
    sp = grid.species
    assert np.array_equal(a[..., sp], b[..., sp]), np.abs(a[..., sp] - b[..., sp]).max()
    assert np.array_equal(a, b) and np.array_equal(a, c)
    with pytest.raises(ValueError):
        split.put_fluxes(blocks[0], 1, split.get_fluxes(blocks[0], 1)[:, :8])
    for h in (fused, split, both):
        h.close()


@pytest.mark.gpu
def test_replaced_mass_scalar_flux_changes_the_two_adjacent_cells():
    """A mass scalar (not renormalised) is linear in its fluxes: a face flux
    raised by dF changes X of the cells beside the face by -+ dt dF/(dx rho)
    and nothing else; the hydro variables do not move."""
    grid, unk, params = make_case("sod2d_rot", nspecies=1, nmass_scalars=1)
    h0, h1 = Hydro(params, grid), Hydro(params, grid)
    for h in (h0, h1):
        h.upload(unk)
    dt, _ = h0.compute_dt()
    blk = 5
    for h in (h0, h1):
        h.compute_fluxes([blk], dt, abi.UPDATE_NONE)
    flx = h1.get_fluxes(blk, 1)
    nx = grid.nb[0] + 1
    i, j, dF = 3, 2, 1e-3
    flx[j * nx + i, 9] += dF                                  # the mass scalar's flux at x face (i, j)
    h1.put_fluxes(blk, 1, flx)
    for h in (h0, h1):
        h.update_solution([blk], dt)
    a, b = _state(h0, grid), _state(h1, grid)
    ms = grid.species.start + 1
    diff = b[..., ms] - a[..., ms]
    rho = a[..., VAR["dens"]]
    dtdx = dt / grid.delta[0]
    assert abs(diff[blk, 0, j, i - 1] + dtdx * dF / rho[blk, 0, j, i - 1]) <= 1e-12
    assert abs(diff[blk, 0, j, i] - dtdx * dF / rho[blk, 0, j, i]) <= 1e-12
    diff[blk, 0, j, i - 1] = diff[blk, 0, j, i] = 0.0
    assert np.all(diff == 0.0)
    assert np.array_equal(np.delete(a, ms, axis=-1), np.delete(b, ms, axis=-1))
    for h in (h0, h1):
        h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_ring", "quad2d_16", "sod2d_reflect", "kh3d_ring"])
def test_amr_species_match_oracle(case):
    """Species on AMR hierarchies: restriction, guard cells (prolonged in
    per-mass form), the species flux register at fine/coarse faces: every
    leaf variable equal to the oracle bit for bit (FP64)."""
    from tests.test_gpu_amr import _run_amr, amr_case, VARS
    from flash5_b200.grid import VAR
    grid, unk, params = amr_case(case, nspecies=2, nmass_scalars=1)
    grid, ref, out, steps = _run_amr(grid, unk, params, 4)
    leaves = grid.leaf_ids
    a, b = grid.interior(out)[leaves], grid.interior(ref)[leaves]
    sp = grid.species
    assert np.array_equal(a[..., sp], b[..., sp]), np.abs(a[..., sp] - b[..., sp]).max()
    for v in VARS:
        assert np.array_equal(a[..., VAR[v]], b[..., VAR[v]]), v


@pytest.mark.gpu
def test_amr_species_regrid_matches_oracle():
    from tests.test_gpu_amr import amr_case
    from flash5_b200.amr import mark_refine_derefine, regrid_native
    grid, unk, params = amr_case("quad2d_16", nspecies=2, nmass_scalars=1)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    _steps(h, o, unk, ref, 2)
    errs = [h.estimate_error("dens", 0.01)]
    lv, pv = errs[0][grid.leaf_ids], errs[0][~grid.is_leaf]
    refine, derefine = mark_refine_derefine(grid, errs, np.quantile(lv, 0.95), np.quantile(pv, 0.7))
    g2, src, how = regrid_native(grid, refine, derefine)
    assert np.any(how == 1) and np.any(how == 2)
    h2 = h.regrid(g2, src, how)
    h.close()
    ref2 = o.regrid(ref, g2, src, how)
    out = g2.new_unk()
    h2.download(out)
    h2.close()
    leaves = g2.leaf_ids
    a, b = g2.interior(out)[leaves], g2.interior(ref2)[leaves]
    assert np.array_equal(a, b), np.abs(a - b).max()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_ring", "kh3d_ring"])
def test_amr_species_mixed_close(case):
    """The mixed path's FP32 species face values on AMR hierarchies (one
    launch per level, species flux register): every scalar within 1e-6
    relative L1 of the FP64 oracle on the leaves, species summing to one."""
    from tests.test_gpu_amr import _run_amr, amr_case
    grid, unk, params = amr_case(case, nspecies=2, nmass_scalars=1, precision=abi.PREC_MIXED)
    grid, ref, out, _ = _run_amr(grid, unk, params, 4)
    leaves = grid.leaf_ids
    a, b = grid.interior(out)[leaves], grid.interior(ref)[leaves]
    sp = grid.species
    l1 = np.abs(a[..., sp] - b[..., sp]).sum(axis=(0, 1, 2, 3)) / np.abs(b[..., sp]).sum(axis=(0, 1, 2, 3))
    assert np.all(l1 <= 1e-6), l1
    assert np.abs(a[..., sp.start] + a[..., sp.start + 1] - 1.0).max() < 1e-13
