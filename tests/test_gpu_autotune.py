"""Launch shapes and the autotuner (marked gpu).

* every candidate launch shape gives the same state and dt bit for bit
  where the candidates share one compiled kernel (threads per CTA of the
  transverse-flux pass and of the FP64 direction kernels: FP64 and mixed,
  HLLC and exact Riemann, 2D and 3D); the mixed direction kernels'
  candidates are separately compiled FMA-contracted kernels, equal to
  rounding (1e-13 of each variable's scale, floor 1);
* autotune leaves the state as it found it, returns one of the candidates
  with a trial per candidate of each knob (the mixed path also the other
  sweep order), and the step after it equals a step with that shape set by
  hand;
* a shape that is not a candidate is refused.
"""
import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.hydro import Hydro, HydroError
from tests.cases import make_case


def _run(h, grid, unk, steps=2):
    h.upload(unk)
    dts = []
    for _ in range(steps):
        dt, loc = h.compute_dt()
        dts.append((dt, loc))
        h(0.0, dt, dt)
    out = grid.new_unk()
    h.download(out)
    return out, dts


@pytest.mark.gpu
@pytest.mark.parametrize("case,prec,rs", [("kh3d", abi.PREC_FP64, abi.RS_HLLC), ("sod2d_rot", abi.PREC_FP64, abi.RS_HLLC),
                                          ("kh3d", abi.PREC_MIXED, abi.RS_HLLC), ("kh3d", abi.PREC_MIXED, abi.RS_EXACT),
                                          ("kh2d_16", abi.PREC_MIXED, abi.RS_HLLC),
                                          ("sod2d_rot", abi.PREC_MIXED, abi.RS_EXACT)])
def test_every_launch_shape_gives_the_same_result(case, prec, rs):
    grid, unk, params = make_case(case, precision=prec, riemann_solver=rs)
    h = Hydro(params, grid)
    ref, ref_dts = _run(h, grid, unk)
    cand = h.tuning_candidates()
    knob = "mx_threads" if prec == abi.PREC_MIXED else "dir_threads"
    shapes = [{knob: v} for v in cand[knob]] + [{"sig_threads": v} for v in cand["sig_threads"]]
    default = h.tuning
    for shape in shapes:
        h.tuning = dict(default, **shape)
        assert h.tuning == dict(default, **shape)
        got, dts = _run(h, grid, unk)
        if "mx_threads" in shape:
            assert [d[1] for d in dts] == [d[1] for d in ref_dts], shape
            np.testing.assert_allclose([d[0] for d in dts], [d[0] for d in ref_dts], rtol=1e-13, atol=0)
            ax = tuple(range(ref.ndim - 1))          # per UNK variable
            # scale floor 1: the transverse velocity of the KH flow is ~0
            lim = 1e-13 * np.maximum(np.abs(ref).max(axis=ax), 1.0)
            assert np.all(np.abs(got - ref).max(axis=ax) <= lim), (shape, np.abs(got - ref).max(axis=ax))
        else:
            assert dts == ref_dts, shape
            assert np.array_equal(got, ref), (shape, np.abs(got - ref).max())
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_autotune_restores_state_and_keeps_a_candidate(prec):
    grid, unk, params = make_case("kh3d", precision=prec)
    h = Hydro(params, grid)
    h.upload(unk)
    dt, _ = h.compute_dt()
    before = grid.new_unk()
    h.download(before)
    best, trials = h.autotune(dt, steps=2)
    after = grid.new_unk()
    h.download(after)
    assert np.array_equal(before, after)
    cand = h.tuning_candidates()
    knob = "mx_threads" if prec == abi.PREC_MIXED else "dir_threads"
    assert best[knob] in cand[knob] and best["sig_threads"] in cand["sig_threads"]
    # the mixed path also tries the other sweep order (kh3d's block counts
    # do not divide by 4, so no runs are offered)
    assert len(trials) == len(cand[knob]) + len(cand["sig_threads"]) + (prec == abi.PREC_MIXED)
    assert all(ms > 0.0 for _, ms in trials)
    assert h.tuning == best
    dt2, loc2 = h.compute_dt()
    assert dt2 == dt
    h(0.0, dt, dt)
    tuned = grid.new_unk()
    h.download(tuned)
    h.close()
    g = Hydro(params, grid)
    g.tuning = best
    g.upload(unk)
    g(0.0, dt, dt)
    manual = grid.new_unk()
    g.download(manual)
    g.close()
    assert np.array_equal(tuned, manual)


@pytest.mark.gpu
def test_non_candidate_shape_is_refused():
    grid, unk, params = make_case("kh3d")
    h = Hydro(params, grid)
    for bad in ({"sig_threads": 100}, {"dir_threads": 1024}, {"mx_threads": 200}):
        with pytest.raises(HydroError):
            h.tuning = dict(h.tuning, **bad)
    h.close()
