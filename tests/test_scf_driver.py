"""The host SCF driver pieces (dft-zig_b200/scf.py) on the CPU, with the oracle as the backend."""
import importlib
import math

import numpy as np
import pytest

import dftzig_loader
from tests.helpers import OracleBackend

dftzig_loader.load()
scf = importlib.import_module("dftzig_b200.scf")
system = importlib.import_module("dftzig_b200.system")


def test_lda_pz_potential_is_derivative():
    n = np.array([1e-4, 1e-3, 0.01, 0.05, 0.2, 1.0])  # both r_s branches
    h = 1e-7 * n
    f_p, _ = scf.lda_pz(n + h)
    f_m, _ = scf.lda_pz(n - h)
    _, v = scf.lda_pz(n)
    assert np.allclose((f_p - f_m) / (2 * h), v, rtol=1e-6)
    f0, v0 = scf.lda_pz(np.array([0.0, 1e-13]))
    assert (f0 == 0).all() and (v0 == 0).all()


def test_ewald_graphene_golden():
    """src/tests.zig:859-870: graphene (c = 20 A) ion-ion energy 50.1056 Ha (ABINIT) within 1%."""
    a, c = 4.6487262675, 37.7945225
    cell = np.array([[a, 0.0, 0.0], [a * 0.5, a * math.sqrt(3.0) / 2.0, 0.0], [0.0, 0.0, c]])
    pos = np.array([[0.0, 0.0, 0.0], [3.0991508450, 2.6839433578, 0.0]])
    e_ha = scf.ewald_energy(cell, np.array([4.0, 4.0]), pos) / 2.0
    assert abs(e_ha - 50.1056) / 50.1056 < 0.01


def test_ewald_cscl_madelung_and_forces():
    """The cell of the reference's Ewald force tests (ewald/ewald.zig:608-700): charges +1 / -1 at the
    corner and the body centre of a 5 bohr cube.  Its energy is the CsCl Madelung energy
    -alpha / d Ha per cell (alpha = 1.762675, d = a sqrt(3) / 2); the forces, taken off the symmetric
    site, are minus the finite-difference energy gradient (h = 1e-5) and sum to zero."""
    a = 5.0
    cell = np.eye(3) * a
    z = np.array([1.0, -1.0])
    pos = np.array([[0.0, 0.0, 0.0], [a / 2, a / 2, a / 2]])
    e_ha = scf.ewald_energy(cell, z, pos) / 2.0
    assert abs(e_ha - (-1.76267477307099 / (a * math.sqrt(3.0) / 2.0))) < 1e-10
    pos = pos + np.array([[0.0, 0.0, 0.0], [0.31, -0.12, 0.05]])
    f = scf.ewald_forces(cell, z, pos)
    h = 1e-5
    for atom in range(2):
        for d in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[atom, d] += h
            pm[atom, d] -= h
            fd = -(scf.ewald_energy(cell, z, pp) - scf.ewald_energy(cell, z, pm)) / (2 * h)
            assert abs(f[atom, d] - fd) < 1e-6 * max(1.0, abs(fd))
    assert np.abs(f.sum(axis=0)).max() < 1e-10


def test_ewald_independent_of_split():
    c = system.crystal("si8")
    z = np.array([4.0] * 8)
    e1 = scf.ewald_energy(c.cell, z, c.positions)
    # a translated copy has the same energy
    e2 = scf.ewald_energy(c.cell, z, c.positions + 0.37)
    assert abs(e1 - e2) < 1e-9 * abs(e1)


def test_ewald_split_parameter_does_not_change_the_energy():
    """The Ewald energy for three split parameters (the default grows with the atom density)."""
    c = system.crystal("si64")
    z = np.array([4.0] * len(c.atom_species))
    e0 = scf.ewald_energy(c.cell, z, c.positions)
    for eta in (0.12, 0.3):
        assert abs(scf.ewald_energy(c.cell, z, c.positions, eta=eta) - e0) < 1e-10 * abs(e0)


def test_pulay_mixer_solves_linear_fixed_point():
    rng = np.random.default_rng(0)
    A = rng.normal(size=(6, 6)) * 0.1
    b = rng.normal(size=6)
    x = np.zeros(6)
    mix = scf.PulayMixer(8)
    for _ in range(30):
        fx = A @ x + b  # fixed point x = A x + b
        x = mix.mix(x, fx - x, 0.5)
    assert np.abs(A @ x + b - x).max() < 1e-9


def test_scf_converges_with_oracle_backend():
    """Si2, 8 Ry, 2x2x2 mesh, fixed occupations: the synthetic Si is a semiconductor (one s-like
    state under a p-like triplet at Gamma) and the potential-mixing loop converges."""
    c = system.crystal("si2")
    p = scf.ScfParams(ecut=8.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-8, iterative_max_iter=100, iterative_tol=1e-9, warmup_steps=0)
    r = scf.run_scf(c, p, OracleBackend())
    assert r.converged
    assert r.iterations < 25
    assert math.isfinite(r.energy) and -9.0 < r.energy_per_atom < -7.0
    g = r.eigenvalues[0]
    assert abs(g[1] - g[3]) < 1e-6 and g[4] - g[3] > 0.02  # occupied triplet, gap above it


def test_model_dielectric_preconditioner_keeps_the_fixed_point():
    """The Pulay residual scaled by P(G) = (l^2 G^2 + 1/eps) / (l^2 G^2 + 1) (the reference's
    apply_model_dielectric_preconditioner, mixing.zig:319-337) changes the path, not the answer: Si2
    with diemac = 12 converges to the energy of the plain run."""
    c = system.crystal("si2")
    base = dict(ecut=8.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-9, iterative_max_iter=100, iterative_tol=1e-10, warmup_steps=0)
    plain = scf.run_scf(c, scf.ScfParams(**base), OracleBackend())
    diel = scf.run_scf(c, scf.ScfParams(**base, diemac=12.0, dielng=1.0), OracleBackend())
    assert plain.converged and diel.converged
    assert abs(plain.energy_per_atom - diel.energy_per_atom) < 1e-8


def test_mixed_backend_switch_rule():
    """GpuBackend("mixed") leaves the reduced-precision contexts when the density residual falls below
    switch_drho, or when it has stopped reaching a new minimum for `stall` observations once it is
    below 10 x switch_drho; a residual that rises above that band is the mixing's own transient and
    does not count."""
    b = scf.GpuBackend(None, "mixed", switch_drho=1e-4, stall=3)
    for d in (1e-2, 3e-2, 5e-2, 2e-3):  # rises above the band: no stall counted
        b.observe(d)
    assert b.use32 and b.since_best == 0
    for d in (9e-4, 9.5e-4, 9.6e-4):
        b.observe(d)
    assert b.use32 and b.since_best == 2
    b.observe(9.7e-4)  # the third observation without a new minimum inside the band
    assert not b.use32 and b.switched_at == 8

    b = scf.GpuBackend(None, "mixed", switch_drho=1e-4, stall=3)
    b.observe(5e-3)
    b.observe(8e-5)  # below the threshold: switch at once
    assert not b.use32 and b.switched_at == 2

    b = scf.GpuBackend(None, "fp64")
    b.observe(1e-9)
    assert not b.use32 and b.switched_at is None
