"""The error norms of the benchmark reports (flash5_b200/metrics.py), the two
comparisons of FLASH's sfocu: L1 relative sum|a-b|/sum|b| and the magnitude
error max|a-b|/max|b|, per conserved variable."""
import numpy as np

from flash5_b200.grid import VAR
from flash5_b200.metrics import conserved, conserved_l1, conserved_linf, l1_rel, mag_err


def test_norms_of_known_differences():
    b = np.array([1.0, -2.0, 3.0, 4.0])
    a = b + np.array([0.0, 0.5, 0.0, -1.0])
    assert l1_rel(a, b) == 1.5 / 10.0
    assert mag_err(a, b) == 1.0 / 4.0
    assert l1_rel(b, b) == 0.0 and mag_err(b, b) == 0.0
    z = np.zeros(3)
    assert l1_rel(z + 1.0, z) == 3.0 and mag_err(z + 1.0, z) == 1.0   # zero reference: absolute norms


def test_conserved_variables_and_their_norms():
    rng = np.random.default_rng(3)
    unk = rng.uniform(0.5, 2.0, size=(2, 1, 4, 4, len(VAR)))
    c = conserved(unk, VAR)
    assert np.array_equal(c["xmom"], unk[..., VAR["dens"]] * unk[..., VAR["velx"]])
    assert np.array_equal(c["ener"], unk[..., VAR["dens"]] * unk[..., VAR["ener"]])
    other = unk.copy()
    other[0, 0, 1, 2, VAR["dens"]] *= 1.0 + 1e-6
    l1, linf = conserved_l1(other, unk, VAR), conserved_linf(other, unk, VAR)
    assert set(l1) == set(linf) == {"dens", "xmom", "ymom", "zmom", "ener"}
    for k in l1:
        assert 0.0 < l1[k] < linf[k] <= 1e-6
