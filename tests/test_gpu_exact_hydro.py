"""Hydro step with the exact Riemann solver (marked gpu).

FLASH5's unsplit path has no exact solver, so these faces are checked
against the oracle's FP64 exact solver (Toro ch. 4, oracle/oracle_exact.c)
inside the same oracle hydro step:

* FP64 path: Newton to 1e-12 on both sides, so the step agrees with the
  oracle to the solver tolerance (CUDA's and glibc's pow differ in the last
  place), not bit for bit: relative L1 <= 1e-10 per conserved variable;
* mixed path (FP32 reconstruction, FP64 solve and update): <= 1e-6;
* learned guess: after training on face states harvested from the hydro
  run itself (faces with strong waves, where the network is consulted),
  the converged fluxes are those of the two-rarefaction start, to the
  solver tolerance (<= 1e-10), in 2D and 3D.
"""
import numpy as np
import pytest

from flash5_b200 import abi, setups
from flash5_b200.grid import UniformGrid, VAR
from flash5_b200.hydro import Hydro, next_dt
from tests.cases import make_case
from tests.test_gpu_parity import conserved_l1, run_pair


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d_rot", "quad2d_16", "sod2d_reflect", "kh3d", "sod3d_rot"])
def test_exact_fp64_matches_oracle(case):
    grid, ref, out, steps = run_pair(case, riemann_solver=abi.RS_EXACT)
    for k, l1 in conserved_l1(out, ref, grid).items():
        assert l1 <= 1e-10, (k, l1)
    for dto, loco, dtg, locg in steps:
        assert abs(dtg - dto) <= 1e-10 * dto


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d_rot", "kh2d_16", "quad2d_16", "kh3d", "sod3d_rot"])
def test_exact_mixed_close(case):
    grid, ref, out, _ = run_pair(case, riemann_solver=abi.RS_EXACT, precision=abi.PREC_MIXED)
    for k, l1 in conserved_l1(out, ref, grid).items():
        assert l1 <= 1e-6, (k, l1)


def _run(h, unk, nsteps, dt0):
    h.upload(unk)
    t, dt, dt_old = 0.0, dt0, dt0
    for _ in range(nsteps):
        h(t + dt, dt, dt_old)
        t += dt
        dtc, _ = h.compute_dt()
        dt_old, dt = dt, next_dt(dtc, dt)
    out = np.zeros_like(unk)
    h.download(out)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [2, 3])
def test_learned_guess_hydro_unchanged(ndim):
    import torch
    from flash5_b200.riemann import ExactRiemann
    if ndim == 2:
        grid = UniformGrid(2, (16, 16), (8, 8), bc="outflow")
        unk = setups.four_quadrant(grid)
        gamma = 1.4
    else:
        grid = UniformGrid(3, (8, 8, 8), (4, 4, 4), bc="outflow")
        unk = setups.sod(grid, xangle=30.0, yangle=70.0)
        gamma = 1.4
    p = abi.default_params(gamma=gamma, riemann_solver=abi.RS_EXACT, precision=abi.PREC_MIXED)
    pl = abi.default_params(gamma=gamma, riemann_solver=abi.RS_EXACT, precision=abi.PREC_MIXED, learned_guess=1)
    h = Hydro(p, grid)
    h.upload(unk)
    dt0, _ = h.compute_dt()
    # harvest face states from the run itself and train the guess on them
    h.harvest(400000, keep_log2=0)
    _run(h, unk, 3, dt0)
    S = h.harvest_fetch(torch)
    h.harvest(0)
    # faces with strong waves and an inexact two-rarefaction guess
    assert S.shape[0] == 7 and S.shape[1] > 500
    Sh = S.cpu().numpy()
    assert np.all(Sh[0] > 0) and np.all(Sh[3] > 0) and np.all(Sh[2] > 0) and np.all(Sh[5] > 0)
    assert np.all(Sh[6] == gamma)
    rs = ExactRiemann(0)
    try:
        loss, ns = rs.fit(S, epochs=30, batch=128)
        assert np.isfinite(loss) and ns > 400
        w = rs.weights()
    finally:
        rs.close()
    ref = _run(h, unk, 4, dt0)
    h.close()
    hl = Hydro(pl, grid)
    hl.set_guess_weights(w)
    got = _run(hl, unk, 4, dt0)
    hl.sync()
    hl.close()
    for k, l1 in conserved_l1(got, ref, grid).items():
        assert l1 <= 1e-10, (k, l1)
