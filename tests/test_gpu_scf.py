"""The SCF driver with the hot path on the GPU against the same driver on the oracle:
total energy per atom within 1e-8 Ry and every eigenvalue within 1e-7 Ry (the plain-FP64 bar)."""
import importlib

import numpy as np
import pytest

import dftzig_loader
from tests.helpers import OracleBackend

pytestmark = pytest.mark.gpu


def test_si2_scf_gpu_matches_oracle(dz):
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si2")
    p = scf.ScfParams(ecut=20.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-8, iterative_max_iter=200, iterative_tol=1e-10, warmup_steps=0, max_iter=40)
    gpu = scf.GpuBackend(dz)
    r_gpu = scf.run_scf(c, p, gpu)
    gpu.close()
    r_ref = scf.run_scf(c, p, OracleBackend())
    assert r_gpu.converged and r_ref.converged
    assert abs(r_gpu.energy_per_atom - r_ref.energy_per_atom) < 1e-8
    for a, b in zip(r_gpu.eigenvalues, r_ref.eigenvalues):
        assert np.abs(np.asarray(a) - np.asarray(b)).max() < 1e-7


def test_al4_smeared_scf_gpu_matches_oracle(dz):
    """Al4 (metal, 27^3 box, odd extents), Fermi-Dirac 0.02 Ry, Fermi level by bisection."""
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("al4")
    p = scf.ScfParams(ecut=15.0, kmesh=(2, 2, 2), nbands=12, convergence=1e-8, iterative_max_iter=200, iterative_tol=1e-10, warmup_steps=0, max_iter=40, smearing=0.02)
    gpu = scf.GpuBackend(dz)
    r_gpu = scf.run_scf(c, p, gpu)
    gpu.close()
    r_ref = scf.run_scf(c, p, OracleBackend())
    assert r_gpu.converged and r_ref.converged
    assert abs(r_gpu.energy_per_atom - r_ref.energy_per_atom) < 1e-8


def test_many_cell_scf_matches_single_runs(dz):
    """run_scf_many (every cell's k-points in one lockstep eigensolver batch per SCF iteration) gives
    the same converged energies as one run_scf per cell."""
    import importlib

    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    cells = [system.crystal("sige8", 2900 + i) for i in range(3)]
    p = scf.ScfParams(ecut=10.0, kmesh=(1, 1, 1), nbands=20, convergence=1e-8, iterative_tol=1e-9,
                      iterative_max_iter=100, warmup_steps=0, smearing=0.01, max_iter=60)
    many, _ = scf.run_scf_many(dz, cells, p)
    for c, r in zip(cells, many):
        b = scf.GpuBackend(dz)
        one = scf.run_scf(c, p, b)
        b.close()
        assert r.converged and one.converged
        assert abs(r.energy_per_atom - one.energy_per_atom) < 1e-8
