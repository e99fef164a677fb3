"""Exact Riemann solver and its learned initial guess on the GPU (marked gpu).

* the device generator matches its numpy replica;
* two-rarefaction-guess solves match the CPU oracle (orc_star_batch) and the
  mpmath golden star states;
* the hand-written training kernel's gradient matches the float64 analytic
  gradient of the reference MLP (which itself matches finite differences in
  tests/test_mlp_ref.py);
* the tensor-core BF16 inference (tcgen05 with TMEM accumulators, the
  default) matches a BF16 numpy forward pass, and the per-warp mma.sync form
  to rounding, on full and partial 128-interface tiles;
* after training on solver-harvested states, Newton from the learned guess
  gives the same p* (to 1e-11) in fewer iterations than from the
  two-rarefaction guess.
"""
import json
import os

import numpy as np
import pytest

from oracle import mlp_ref, orc

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def rs():
    from flash5_b200.riemann import ExactRiemann
    r = ExactRiemann(0)
    yield r
    r.close()


@pytest.mark.gpu
def test_generator_matches_replica(rs):
    S = rs.generate(2024, 5000).cpu().numpy()
    idx = [0, 1, 2, 17, 999, 4999]
    ref = mlp_ref.generate(2024, idx)
    np.testing.assert_allclose(S[:, idx], ref, rtol=1e-13, atol=0)


@pytest.mark.gpu
def test_two_rarefaction_solves_match_oracle(rs):
    n = 20000
    S = rs.generate(11, n)
    out, iters, flags = rs.solve(S, learned=False)
    torch = rs.torch
    torch.cuda.synchronize()
    assert rs.sync() == 0
    h = S.cpu().numpy()
    ps, us, it, st = orc.star_batch(*h, tol=1e-12, max_iter=50)
    o = out.cpu().numpy()
    fl = flags.cpu().numpy()
    vac = st == 2
    assert np.array_equal(vac, (fl & 2) != 0)
    ok = ~vac
    assert np.all(st[ok] == 0)
    np.testing.assert_allclose(o[0][ok], ps[ok], rtol=1e-11)
    np.testing.assert_allclose(o[1][ok], us[ok], rtol=1e-9, atol=1e-9 * np.abs(h[1][ok]).max())


@pytest.mark.gpu
def test_golden_star_states(rs):
    cases = json.load(open(os.path.join(GOLD, "riemann_star.json")))["cases"]
    S = np.array([[c["dl"], c["ul"], c["pl"], c["dr"], c["ur"], c["pr"], c["gamma"]] for c in cases]).T.copy()
    St = rs.torch.tensor(S, device="cuda:0")
    out, _, _ = rs.solve(St, learned=False)
    o = out.cpu().numpy()
    for k, c in enumerate(cases):
        assert abs(o[0][k] / float(c["pstar"]) - 1) < 1e-11, (c, o[0][k])
        assert abs(o[1][k] - float(c["ustar"])) < 1e-10 * max(1.0, abs(float(c["ustar"])))


@pytest.mark.gpu
def test_gradient_matches_reference(rs):
    torch = rs.torch
    rng = np.random.default_rng(3)
    w = (rng.normal(size=mlp_ref.NPARAM) * 0.3).astype(np.float32)
    rs.set_weights(w)
    n = 300
    X = rng.normal(size=(n, 8)).astype(np.float32)
    T = rng.normal(size=n).astype(np.float32)
    Xd, Td = torch.tensor(X, device="cuda:0"), torch.tensor(T, device="cuda:0")
    idx = torch.arange(n, dtype=torch.int32, device="cuda:0")
    g, loss = rs.grad(Xd, Td, idx)
    lref, gref = mlp_ref.loss_and_grad(w.astype(np.float64), X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    for lo, hi in [(mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
                   (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.NPARAM)]:
        scale = np.abs(gref[lo:hi]).max()
        assert np.abs(g[lo:hi] - gref[lo:hi]).max() <= 1e-4 * scale + 1e-7, (lo, hi)


@pytest.mark.gpu
def test_tensor_core_inference_matches_bf16_reference(rs):
    rng = np.random.default_rng(5)
    w = (rng.normal(size=mlp_ref.NPARAM) * 0.3).astype(np.float32)
    rs.set_weights(w)
    S = rs.generate(99, 4096)
    y = rs.predict(S).cpu().numpy()
    h = S.cpu().numpy()
    dl, ul, pl, dr, ur, pr, g = h
    cl, cr = np.sqrt(g * pl / dl), np.sqrt(g * pr / dr)
    ok = ~(2 * (cl + cr) / (g - 1) <= ur - ul)
    f, _ = mlp_ref.features(h[:, ok])
    yb = mlp_ref.forward_bf16(w, f.astype(np.float32))
    y64, _, _ = mlp_ref.forward(w, f)
    err = np.abs(y[ok] - yb)
    assert err.mean() < 2e-2 * (1 + np.abs(yb).mean()), err.mean()
    # the BF16 network is a usable approximation of the FP64 one
    assert np.abs(y[ok] - y64).mean() < 0.1 * (1 + np.abs(y64).mean())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 129, 4096 + 37])
def test_tcgen05_inference_matches_warp_mma(rs, n):
    from flash5_b200.riemann import INFER_TCGEN05, INFER_WARP_MMA
    rng = np.random.default_rng(7)
    w = (rng.normal(size=mlp_ref.NPARAM) * 0.3).astype(np.float32)
    rs.set_weights(w)
    S = rs.generate(123, n)
    try:
        rs.set_inference(INFER_WARP_MMA)
        yw = rs.predict(S).cpu().numpy()
        rs.set_inference(INFER_TCGEN05)
        yt = rs.predict(S).cpu().numpy()
    finally:
        rs.set_inference(INFER_TCGEN05)
    assert rs.sync() == 0
    assert np.all(np.isfinite(yt))
    d = np.abs(yt - yw) / (1.0 + np.abs(yw))
    # same BF16 operands and FP32 accumulation (the tcgen05 form takes the
    # FP32 biases and w3 as two BF16 parts); a hidden unit's BF16 rounding
    # can flip with the accumulation order, nothing more
    assert d.max() <= 2e-2, d.max()
    assert np.median(d) <= 1e-4, np.median(d)


@pytest.mark.gpu
def test_inference_mode_rejects_unknown_values(rs):
    from flash5_b200.riemann import RiemannError
    with pytest.raises(RiemannError):
        rs.set_inference(7)


@pytest.mark.gpu
def test_learned_guess_same_result_fewer_iterations(rs):
    torch = rs.torch
    from flash5_b200.riemann import ExactRiemann
    r = ExactRiemann(0)                       # fresh He-initialised network
    try:
        Str = r.generate(1, 2000000)
        out, _, _ = r.solve(Str, learned=False)
        X, T, ns = r.make_samples(Str, out)
        loss = r.train(X, T, ns, epochs=8, batch=4096, lr=2e-3)
        assert np.isfinite(loss)
        S = r.generate(2, 200000)
        o0, it0, f0 = r.solve(S, learned=False)
        o1, it1, f1 = r.solve(S, learned=True)
        from flash5_b200.riemann import INFER_TCGEN05, INFER_WARP_MMA
        r.set_inference(INFER_WARP_MMA)
        o2, it2, f2 = r.solve(S, learned=True)
        r.set_inference(INFER_TCGEN05)
        torch.cuda.synchronize()
        assert r.sync() == 0
        # the tcgen05 and per-warp network starts converge to the same p*
        ok2 = (f2.cpu().numpy() & 2) == 0
        p2 = o2[0].cpu().numpy()
        assert np.array_equal(ok2, (f1.cpu().numpy() & 2) == 0)
        assert (np.abs(p2[ok2] - o1[0].cpu().numpy()[ok2]) / p2[ok2]).max() <= 1e-11
        p0, p1 = o0[0].cpu().numpy(), o1[0].cpu().numpy()
        fl0, fl1 = f0.cpu().numpy(), f1.cpu().numpy()
        ok = (fl0 & 2) == 0
        assert np.array_equal(fl0 & 2, fl1 & 2)
        assert np.all((fl0[ok] & 4) == 0) and np.all((fl1[ok] & 4) == 0)
        rel = np.abs(p1[ok] - p0[ok]) / p0[ok]
        assert rel.max() <= 1e-11, rel.max()
        m0, m1 = it0.cpu().numpy()[ok].mean(), it1.cpu().numpy()[ok].mean()
        assert m1 < m0, (m0, m1)
        assert ((fl1[ok] & 1) != 0).mean() < 0.1
    finally:
        r.close()
