"""The split step (marked gpu): flash_hy_compute_fluxes / get / put /
flash_hy_update_solution, the form of hy_computeFluxes (Uout disassociated)
and hy_updateSolution that FLASH wraps around its own flux correction.

* the FP64 fluxes of a block equal the oracle's face fluxes bit for bit, in
  FLASH's flx(NFLUXES, i, j, k) layout;
* compute_fluxes(UPDATE_NONE) leaves the state alone, and the update from
  the kept fluxes equals the fused step on the same blocks bit for bit
  (FP64 and mixed), as does compute_fluxes(UPDATE_ALL);
* a replaced face flux changes exactly the two cells beside the face, by
  -+ dt/dx times the change (the conservative update is linear in the
  fluxes).
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro
from oracle import orc
from tests.cases import make_case


def _state(h, grid):
    out = grid.new_unk()
    h.download(out)
    return grid.interior(out).copy()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d_rot", "kh3d"])
def test_block_fluxes_match_oracle(case):
    grid, unk, params = make_case(case)
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
        for d in range(grid.ndim):
            got = h.get_fluxes(b, d + 1)
            assert np.array_equal(got, want[d]), (b, d, np.abs(got - want[d]).max())
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case,prec", [("sod2d_rot", abi.PREC_FP64), ("kh3d", abi.PREC_FP64),
                                       ("kh3d", abi.PREC_MIXED), ("kh2d_16", abi.PREC_MIXED)])
def test_split_step_equals_fused_step(case, prec):
    grid, unk, params = make_case(case, precision=prec)
    blocks = list(range(grid.nblocks))[::2]
    fused, split, both = Hydro(params, grid), Hydro(params, grid), Hydro(params, grid)
    for h in (fused, split, both):
        h.upload(unk)
    dt, _ = fused.compute_dt()
    before = _state(split, grid)
    fused.step_blocks(blocks, dt, dt, dt)
    split.compute_fluxes(blocks, dt, abi.UPDATE_NONE)
    assert np.array_equal(_state(split, grid), before)         # Uout disassociated: no update
    split.update_solution(blocks, dt)
    both.compute_fluxes(blocks, dt, abi.UPDATE_ALL)
    a, b, c = _state(fused, grid), _state(split, grid), _state(both, grid)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    # the kept fluxes survive a get/put round trip
    for blk in blocks[:2]:
        for d in range(1, grid.ndim + 1):
            split.put_fluxes(blk, d, split.get_fluxes(blk, d))
    for h in (fused, split, both):
        h.close()


@pytest.mark.gpu
def test_replaced_flux_changes_the_two_adjacent_cells():
    grid, unk, params = make_case("sod2d_rot")
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
    flx[j * nx + i, 0] += dF                                  # mass flux of x face (i, j)
    h1.put_fluxes(blk, 1, flx)
    for h in (h0, h1):
        h.update_solution([blk], dt)
    a, b = _state(h0, grid), _state(h1, grid)
    diff = b[..., VAR["dens"]] - a[..., VAR["dens"]]
    dtdx = dt / grid.delta[0]
    assert abs(diff[blk, 0, j, i - 1] + dtdx * dF) <= 1e-12 and abs(diff[blk, 0, j, i] - dtdx * dF) <= 1e-12
    diff[blk, 0, j, i - 1] = diff[blk, 0, j, i] = 0.0
    assert np.all(diff == 0.0)
    for h in (h0, h1):
        h.close()
