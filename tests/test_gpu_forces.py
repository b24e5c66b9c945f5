"""Hellmann-Feynman forces on the device (dftcuda_local_forces, dftcuda_nonlocal_forces) against the
oracle (oracle/forces.py), and the SCF driver's total forces against a finite difference of the
converged total energy."""
import importlib
import math

import numpy as np
import pytest

from oracle import forces as of
from oracle import potential as op

pytestmark = pytest.mark.gpu


def _mods():
    return importlib.import_module("dftzig_b200.scf"), importlib.import_module("dftzig_b200.system")


def test_local_forces_match_oracle(dz):
    _, system = _mods()
    c = system.crystal("si8")
    ecut = 10.0
    dims = system.fft_box(ecut, c.recip)
    gth = [[4.0, 0.44, -7.3, 1.1, -0.2, 0.03], [3.0, 0.5, -6.0, 0.0, 0.4, 0.0]]
    rng = np.random.default_rng(8)
    sp = rng.integers(0, 2, len(c.atom_species)).astype(np.int32)
    pos = np.asarray(c.positions) + rng.normal(scale=0.2, size=np.shape(c.positions))
    N = dims[0] * dims[1] * dims[2]
    g2 = op.g2_table(dims, c.recip)
    rho = 0.02 + 0.01 * op.to_r(np.where(g2 < 4.0, op.to_g(rng.normal(size=N), dims), 0.0), dims)
    pc = dz.PotentialContext(dims, c.volume, c.recip, history=1)
    try:
        for g2max in (0.0, 4 * ecut):
            ref = of.local_forces(rho, gth, sp, pos, dims, c.recip, g2max)
            got = pc.local_forces(gth, sp, pos, rho, g2max)
            assert np.abs(got - ref).max() < 1e-10 * max(1.0, np.abs(ref).max())
    finally:
        pc.close()


def test_local_forces_radial_match_oracle(dz):
    """Local forces with the radial-mesh form factor (dftcuda_local_forces_radial) against the oracle,
    two species, displaced atoms, with and without the |G|^2 cut."""
    _, system = _mods()
    c = system.crystal("si8")
    ecut = 10.0
    dims = system.fft_box(ecut, c.recip)
    rng = np.random.default_rng(9)
    sp = rng.integers(0, 2, len(c.atom_species)).astype(np.int32)
    pos = np.asarray(c.positions) + rng.normal(scale=0.2, size=np.shape(c.positions))
    meshes = [system.species("Si").mesh, system.species("Ge").mesh]
    N = dims[0] * dims[1] * dims[2]
    g2 = op.g2_table(dims, c.recip)
    rho = 0.02 + 0.01 * op.to_r(np.where(g2 < 4.0, op.to_g(rng.normal(size=N), dims), 0.0), dims)
    pc = dz.PotentialContext(dims, c.volume, c.recip, history=1)
    try:
        for g2max in (0.0, 4 * ecut):
            ref = of.local_forces_radial(rho, meshes, sp, pos, dims, c.recip, g2max)
            got = pc.local_forces_radial(meshes, sp, pos, rho, g2max)
            assert np.abs(got - ref).max() < 1e-10 * max(1.0, np.abs(ref).max())
    finally:
        pc.close()


def test_nonlocal_forces_match_oracle(dz):
    scf, system = _mods()
    c = system.crystal("si2")
    inp = system.kpoint_inputs(c, 12.0, (0.25, 0.0, 0.125))
    pos = np.asarray(c.positions, dtype=np.float64) + np.array([[0.03, -0.02, 0.05], [0.0, 0.01, -0.04]])
    kc = dz.KpointContext(*inp.dims, inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, 0)
    try:
        kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, pos)
        rng = np.random.default_rng(9)
        n = inp.basis.hkl.shape[0]
        vecs = rng.normal(size=(5, n)) + 1j * rng.normal(size=(5, n))
        w = np.array([0.4, 0.4, 0.2, 0.0, 0.1])
        ref = of.nonlocal_forces(inp.basis.gcart, inp.species_phi, inp.atom_species, pos, vecs, w, c.volume)
        got = kc.nonlocal_forces(vecs, w, len(inp.atom_species))
        assert np.abs(got - ref).max() < 1e-10 * max(1.0, np.abs(ref).max())
    finally:
        kc.close()


def test_scf_forces_match_energy_finite_difference(dz):
    """Si2 with one atom displaced: the resident driver's total force on x of atom 1 against
    -(E(x + h) - E(x - h)) / 2h of fully converged SCF energies (h = 0.005 bohr)."""
    scf, system = _mods()
    base = system.crystal("si2")
    p = scf.ScfParams(ecut=14.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-10, iterative_max_iter=200, iterative_tol=1e-11,
                      warmup_steps=0, max_iter=60)

    def run(dx, forces=False):
        c = system.crystal("si2")
        c.positions = np.asarray(base.positions, dtype=np.float64).copy()
        c.positions[1, 0] += 0.1 + dx
        b = scf.GpuBackend(dz, resident=True)
        r = scf.run_scf(c, p, b, forces=forces)
        b.close()
        assert r.converged
        return r

    r0 = run(0.0, forces=True)
    h = 0.005
    fd = -(run(h).energy - run(-h).energy) / (2 * h)
    assert abs(r0.forces[1, 0] - fd) < 2e-4 + 1e-3 * abs(fd), (r0.forces[1, 0], fd)
    assert abs(r0.forces[1, 0]) > 1e-3  # the displacement produces a real force
    assert np.abs(r0.forces.sum(axis=0)).max() < 1e-3  # no net force beyond grid effects


@pytest.mark.parametrize("name,k", [("si8", (0.13, -0.07, 0.21)), ("sige8", (0.0, 0.25, 0.0))])
def test_nonlocal_stress_matches_oracle(dz, name, k):
    """dftcuda_nonlocal_stress (derivative-projector GEMMs on the device) against the oracle's
    restatement of stress/nonlocal_stress.zig (oracle/stress.py, itself checked as the strain
    derivative of the nonlocal energy): the components a <= b, 1e-10 of the largest."""
    from oracle import stress as ost

    _, system = _mods()
    c = system.crystal(name, 1)
    ecut = 12.0
    tables = [[system.radial_table(sp, i, ecut) for i in range(len(sp.betas))] for sp in c.species]
    inp = system.kpoint_inputs(c, ecut, k, tables=tables)
    kc = dz.KpointContext(*inp.dims, inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart)
    kc.set_vloc(inp.local_r)
    kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
    rng = np.random.default_rng(5)
    nb = 6
    vecs = rng.normal(size=(nb, kc.n)) + 1j * rng.normal(size=(nb, kc.n))
    vecs /= np.linalg.norm(vecs, axis=1, keepdims=True)
    w = np.array([0.5, 0.5, 0.25, 0.0, 0.125, -0.1])
    kpg = inp.basis.kpg
    dphi = [system.projector_derivatives(sp, kpg, tables[s]) for s, sp in enumerate(c.species)]
    got = kc.nonlocal_stress(kpg, dphi, vecs, w)
    species = []
    for s, sp in enumerate(c.species):
        t = tables[s]
        species.append(([l for l, _ in sp.betas], sp.dij, lambda b, q, t=t: system._interp(t[b], q),
                        lambda b, q, t=t: system._interp_deriv(t[b], q)))
    ref = ost.nonlocal_stress(kpg, inp.basis.gcart, species, inp.atom_species, inp.positions, vecs, w, inp.volume)
    kc.close()
    assert np.all(np.tril(got, -1) == 0.0)
    assert np.abs(got - ref).max() < 1e-10 * np.abs(ref).max()
