"""The nonlocal-stress oracle (oracle/stress.py) on the CPU: every component it fills is the strain
derivative of the nonlocal energy at fixed plane-wave coefficients, sigma_ab = (1/Omega) dE/d eps_ba
for the deformation x -> (I + eps) x (finite differences, h = 1e-5), and the angular derivative
d_ylm_dq is the gradient of real_ylm."""
import importlib
import math

import numpy as np
import pytest

import dftzig_loader
from oracle import stress as ost
from oracle.pseudo import real_ylm

dftzig_loader.load()
system = importlib.import_module("dftzig_b200.system")


def _radial(coef, width, l_list):
    def r(b, q):
        l = l_list[b]
        return coef[b] * q**l * np.exp(-width[b] * q * q)

    def dr(b, q):
        l = l_list[b]
        lead = l * q ** (l - 1) if l > 0 else 0.0 * q
        return coef[b] * (lead - 2.0 * width[b] * q ** (l + 1)) * np.exp(-width[b] * q * q)

    return r, dr


@pytest.mark.parametrize("lmax", [1, 2])
def test_d_ylm_dq_is_the_gradient(lmax):
    rng = np.random.default_rng(lmax)
    q = rng.normal(size=(50, 3))
    h = 1e-6
    for m in range(-lmax, lmax + 1):
        g = ost.d_ylm_dq(lmax, m, q)
        for d in range(3):
            e = np.zeros(3)
            e[d] = h
            fd = (real_ylm(lmax, m, *(q + e).T) - real_ylm(lmax, m, *(q - e).T)) / (2 * h)
            np.testing.assert_allclose(g[:, d], fd, atol=1e-8)


def test_nonlocal_stress_is_the_strain_derivative_of_the_energy():
    c = system.crystal("si2")
    k = np.array([0.11, -0.07, 0.05])
    bas = system.basis(c.recip, 6.0, k)
    gcart = np.asarray(bas.hkl, dtype=np.float64) @ np.asarray(c.recip)  # G
    kpg = gcart + k @ np.asarray(c.recip)  # k + G
    rng = np.random.default_rng(11)
    species = []
    for l_list in ([0, 1], [0, 1, 2, 1]):
        nb = len(l_list)
        d = rng.normal(size=(nb, nb))
        d = 0.5 * (d + d.T)
        r, dr = _radial(rng.uniform(0.5, 2.0, nb), rng.uniform(0.2, 0.6, nb), l_list)
        species.append((l_list, d, r, dr))
    atom_species = [0, 1, 1]
    positions = rng.normal(scale=2.0, size=(3, 3))
    nbands = 4
    n = len(kpg)
    vecs = rng.normal(size=(nbands, n)) + 1j * rng.normal(size=(nbands, n))
    weights = np.array([0.5, 0.25, 0.0, 0.125])
    vol = c.volume
    sig = ost.nonlocal_stress(kpg, gcart, species, atom_species, positions, vecs, weights, vol)
    assert np.all(np.tril(sig, -1) == 0.0)  # the reference fills a <= b only
    h = 1e-5
    for a in range(3):
        for b in range(a, 3):
            eps = np.zeros((3, 3))
            eps[b, a] = h
            ep = ost.nonlocal_energy(kpg, gcart, species, atom_species, positions, vecs, weights, vol, eps)
            em = ost.nonlocal_energy(kpg, gcart, species, atom_species, positions, vecs, weights, vol, -eps)
            fd = (ep - em) / (2 * h * vol)
            assert abs(sig[a, b] - fd) <= 1e-6 * np.abs(sig).max(), (a, b, sig[a, b], fd)
    # the unstrained energy is the diagonal term's E_nl: sum_n f_n E_nl,n
    e0 = ost.nonlocal_energy(kpg, gcart, species, atom_species, positions, vecs, weights, vol)
    assert abs(e0) > 0.0
