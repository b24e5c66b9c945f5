"""The force oracle (oracle/forces.py) against finite differences of the energy terms it
differentiates, with the density or wave functions held fixed."""
import importlib
import math

import numpy as np

import dftzig_loader
from oracle import forces as of
from oracle import potential as op

dftzig_loader.load()
scf = importlib.import_module("dftzig_b200.scf")
system = importlib.import_module("dftzig_b200.system")


def test_ewald_forces_are_minus_the_energy_gradient():
    c = system.crystal("si8")
    z = np.array([4.0] * 8)
    pos = c.positions + np.random.default_rng(1).normal(scale=0.1, size=c.positions.shape)
    eta = 0.25
    f = of.ewald_forces(c.cell, z, pos, eta)
    h = 1e-5
    for a, d in [(0, 0), (3, 1), (7, 2)]:
        pp, pm = pos.copy(), pos.copy()
        pp[a, d] += h
        pm[a, d] -= h
        fd = -(scf.ewald_energy(c.cell, z, pp, eta=eta) - scf.ewald_energy(c.cell, z, pm, eta=eta)) / (2 * h)
        assert abs(f[a, d] - fd) < 1e-6 * max(1.0, abs(fd)), (a, d, f[a, d], fd)
    assert np.abs(f.sum(axis=0)).max() < 1e-9  # Newton's third law
    # the driver's own Ewald forces
    np.testing.assert_allclose(scf.ewald_forces(c.cell, z, pos), f, atol=1e-9)


def test_local_forces_are_minus_the_energy_gradient():
    c = system.crystal("si8")
    ecut = 8.0
    dims = system.fft_box(ecut, c.recip)
    gth = [[sp.params["z"], sp.params["rloc"], sp.params["c1"], sp.params["c2"], 0.0, 0.0] for sp in c.species]
    rng = np.random.default_rng(2)
    N = dims[0] * dims[1] * dims[2]
    g2 = op.g2_table(dims, c.recip)
    rho = 0.02 + 0.01 * op.to_r(np.where(g2 < 3.0, op.to_g(rng.normal(size=N), dims), 0.0), dims)
    pos = np.array(c.positions, dtype=np.float64)
    f = of.local_forces(rho, gth, c.atom_species, pos, dims, c.recip, 4 * ecut)

    def energy(p):
        vg, _ = op.ionic_potential(gth, c.atom_species, p, dims, c.recip, c.volume, 4 * ecut)
        return c.volume * float(np.real(np.vdot(vg, op.to_g(rho, dims))))

    h = 1e-5
    for a, d in [(0, 0), (5, 2)]:
        pp, pm = pos.copy(), pos.copy()
        pp[a, d] += h
        pm[a, d] -= h
        fd = -(energy(pp) - energy(pm)) / (2 * h)
        assert abs(f[a, d] - fd) < 1e-6 * max(1.0, abs(fd)), (a, d, f[a, d], fd)


def test_radial_local_forces_are_minus_the_energy_gradient():
    """The radial-mesh local forces (local_force.zig:66-111 with local_vq_short_range) are minus the
    finite-difference gradient of the local energy Omega sum_G Re(V(G)* rho(G)) of the same form."""
    from oracle import pseudo

    c = system.crystal("si8")
    ecut = 8.0
    dims = system.fft_box(ecut, c.recip)
    meshes = [sp.mesh for sp in c.species]
    rng = np.random.default_rng(3)
    N = dims[0] * dims[1] * dims[2]
    g2 = op.g2_table(dims, c.recip)
    rho = 0.02 + 0.01 * op.to_r(np.where(g2 < 3.0, op.to_g(rng.normal(size=N), dims), 0.0), dims)
    pos = np.array(c.positions, dtype=np.float64)
    f = of.local_forces_radial(rho, meshes, c.atom_species, pos, dims, c.recip, 4 * ecut)

    def energy(p):
        vg, _ = pseudo.ionic_potential_radial(meshes, c.atom_species, p, dims, c.recip, c.volume, 4 * ecut)
        return c.volume * float(np.real(np.vdot(vg, op.to_g(rho, dims))))

    h = 1e-5
    for a, d in [(1, 1), (6, 0)]:
        pp, pm = pos.copy(), pos.copy()
        pp[a, d] += h
        pm[a, d] -= h
        fd = -(energy(pp) - energy(pm)) / (2 * h)
        assert abs(f[a, d] - fd) < 1e-6 * max(1.0, abs(fd)), (a, d, f[a, d], fd)


def test_nonlocal_forces_are_minus_the_energy_gradient():
    c = system.crystal("si2")
    ecut = 10.0
    inp = system.kpoint_inputs(c, ecut, (0.25, 0.0, 0.125))
    kpg = inp.basis.gcart
    n = kpg.shape[0]
    rng = np.random.default_rng(3)
    vecs = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    w = np.array([0.5, 0.3, 0.0])
    pos = np.array(c.positions, dtype=np.float64) + 0.05

    def energy(p):
        e = 0.0
        for a, (s, tau) in enumerate(zip(c.atom_species, p)):
            l_list, dij, phi = inp.species_phi[s]
            offs, tot = [], 0
            for l in l_list:
                offs.append(tot)
                tot += 2 * l + 1
            phase = np.exp(1j * (kpg @ tau))
            for b in range(3):
                pr = np.asarray(phi) @ (phase * vecs[b])
                for i, li in enumerate(l_list):
                    for j, lj in enumerate(l_list):
                        if li == lj:
                            for m in range(2 * li + 1):
                                e += w[b] * float(np.real(np.conj(pr[offs[i] + m]) * dij[i][j] * pr[offs[j] + m])) / c.volume
        return e

    f = of.nonlocal_forces(kpg, inp.species_phi, c.atom_species, pos, vecs, w, c.volume)
    h = 1e-6
    for a, d in [(0, 0), (1, 2)]:
        pp, pm = pos.copy(), pos.copy()
        pp[a, d] += h
        pm[a, d] -= h
        fd = -(energy(pp) - energy(pm)) / (2 * h)
        assert abs(f[a, d] - fd) < 1e-6 * max(1e-3, abs(fd)), (a, d, f[a, d], fd)
