"""Fermi level and Fermi-Dirac occupations on the device (dftcuda_fermi_occupations) against the
oracle's restatement of find_fermi_level_spin / smearing_occ / smearing_entropy
(src/features/scf/fermi_level.zig:7-124).

Both run the same bracket-and-bisection schedule; the device sums the electron count in a different
order, so the Fermi levels agree to the bisection's resolution (1e-9 Ry here) and the device's
count at its own Fermi level meets the reference's stop rule |N(mu) - N_e| < 1e-8."""
import numpy as np
import pytest

from oracle import density as odens

pytestmark = pytest.mark.gpu

# (nk, nbands, nelec, sigma): config 2 (8 k, 160 bands, 256 electrons, 0.01 Ry), config 3 (Al4:
# 12 electrons, 0.02 Ry) on a table as long as its IBZ, a gapless toy and the table that spills from
# shared memory to global memory
CASES = [(8, 160, 256.0, 0.01), (260, 12, 12.0, 0.02), (3, 20, 32.0, 0.005), (700, 12, 13.0, 0.02)]


@pytest.mark.parametrize("nk,nb,nelec,sigma", CASES)
def test_fermi_level_matches_oracle(dz, nk, nb, nelec, sigma):
    rng = np.random.default_rng(nk * 1000 + nb)
    values = np.sort(rng.normal(0.4, 0.3, size=(nk, nb)), axis=1)
    w = rng.uniform(0.5, 1.5, size=nk)
    w /= w.sum()
    mu, occ, eb, es = dz.fermi_occupations(values, w, nelec, sigma)
    mu_ref = odens.find_fermi_level(nelec, sigma, w, values)
    assert abs(mu - mu_ref) < 1e-9
    assert abs(odens.electron_count(mu, sigma, w, values) - nelec) < 1e-8
    occ_ref = np.array([[odens.smearing_occ(float(e), mu, sigma) for e in row] for row in values])
    assert np.abs(occ - occ_ref).max() < 1e-14
    eb_ref = sum(2.0 * w[k] * float(np.dot(occ_ref[k], values[k])) for k in range(nk))
    es_ref = sum(2.0 * w[k] * sum(odens.smearing_entropy(float(f)) for f in occ_ref[k]) for k in range(nk))
    assert abs(eb - eb_ref) < 1e-12 * max(1.0, abs(eb_ref))
    assert abs(es - es_ref) < 1e-12 * max(1.0, abs(es_ref))


def test_step_occupations_without_smearing(dz):
    values = np.array([[-0.5, -0.1, 0.2, 0.6]])
    mu, occ, _, es = dz.fermi_occupations(values, [1.0], 4.0, 0.0)  # 2 bands x 2 spins filled
    assert -0.1 <= mu < 0.2
    assert (occ == np.array([[1.0, 1.0, 0.0, 0.0]])).all() and es == 0.0


def test_rejects_empty_table(dz):
    with pytest.raises(dz.InvalidMatrixSize):
        dz.fermi_occupations(np.zeros((0, 4)), [], 1.0, 0.01)
