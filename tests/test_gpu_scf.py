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
    many_dev, _ = scf.run_scf_many(dz, cells, p, resident=True)
    for c, r, rd in zip(cells, many, many_dev):
        b = scf.GpuBackend(dz)
        one = scf.run_scf(c, p, b)
        b.close()
        assert r.converged and one.converged and rd.converged
        assert abs(r.energy_per_atom - one.energy_per_atom) < 1e-8
        assert abs(rd.energy_per_atom - one.energy_per_atom) < 1e-8


@pytest.mark.parametrize("cell,kw", [
    ("si2", dict(ecut=20.0, kmesh=(2, 2, 2), nbands=8)),
    ("al4", dict(ecut=15.0, kmesh=(2, 2, 2), nbands=12, smearing=0.02)),
], ids=["si2", "al4-smeared"])
def test_resident_scf_matches_host_driver(dz, cell, kw):
    """The resident driver (eigenvectors, density, Hartree-XC potential and Pulay history on the
    device: csrc/potential.cu; the per-k inputs built on the device too) against the host-side
    inputs, potential and mixing with the same eigensolver: iterations within two, energy per atom
    within 1e-10 Ry, density within 1e-9 relative.  Converged to 1e-10 so that the two paths, whose
    inputs differ in the last bits (device and host Y_lm), meet at the same fixed point."""
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal(cell)
    p = scf.ScfParams(**kw, convergence=1e-10, iterative_max_iter=200, iterative_tol=1e-11, warmup_steps=0, max_iter=60)
    host = scf.GpuBackend(dz)
    r_host = scf.run_scf(c, p, host)
    host.close()
    dev = scf.GpuBackend(dz, resident=True)
    r_dev = scf.run_scf(c, p, dev)
    dev.close()
    assert r_host.converged and r_dev.converged
    assert abs(r_dev.iterations - r_host.iterations) <= 2
    assert abs(r_dev.energy_per_atom - r_host.energy_per_atom) < 1e-10
    assert np.abs(r_dev.rho - r_host.rho).max() < 1e-9 * np.abs(r_host.rho).max()
    for a, b in zip(r_dev.eigenvalues, r_host.eigenvalues):
        assert np.abs(np.asarray(a) - np.asarray(b)).max() < 1e-9


def test_pbe_scf_converges_and_differs_from_lda(dz):
    """Si2 with the PBE functional (device potential, resident driver) converges; its energy is
    within the usual PBE-LDA spread and its final potential matches the oracle's PBE build."""
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    from oracle import potential as op
    c = system.crystal("si2")
    out = {}
    for xc in ("lda", "pbe"):
        p = scf.ScfParams(ecut=20.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-8, iterative_max_iter=200, iterative_tol=1e-10,
                          warmup_steps=0, max_iter=40, xc=xc)
        b = scf.GpuBackend(dz, resident=True)
        out[xc] = scf.run_scf(c, p, b)
        b.close()
        assert out[xc].converged, xc
    d = out["pbe"].energy_per_atom - out["lda"].energy_per_atom
    assert 1e-3 < abs(d) < 0.5, d
    dims = system.fft_box(20.0, c.recip)
    _, _, e_xc, _ = op.hxc_potential(out["pbe"].rho, dims, c.recip, c.volume, functional="pbe")
    assert abs(out["pbe"].terms["xc"] - e_xc) < 1e-9 * abs(e_xc)


@pytest.mark.parametrize("min_pw", [0, 4096], ids=["tf32x3-contexts", "small-kpoints-fp64"])
def test_mixed_precision_scf_reaches_the_fp64_energy(dz, min_pw):
    """GpuBackend("mixed"): TF32X3 contexts (FP32 FFT passes, split-TF32 tensor-core GEMMs) while the
    density residual is large, FP64 contexts after the switch; the converged energy per atom equals
    the plain FP64 run's within 1e-8 Ry and the switch happened.  With the default threshold Si8's
    k-points (~1,500 plane waves) stay FP64 throughout (no second context), which must also agree."""
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si8")
    p = scf.ScfParams(ecut=20.0, kmesh=(1, 1, 1), nbands=20, convergence=1e-9, max_iter=60)
    b = scf.GpuBackend(dz, resident=True)
    ref = scf.run_scf(c, p, b)
    b.close()
    m = scf.GpuBackend(dz, "mixed", resident=True, min_pw_reduced=min_pw)
    r = scf.run_scf(c, p, m)
    m.close()
    assert ref.converged and r.converged
    assert abs(r.energy_per_atom - ref.energy_per_atom) < 1e-8
    assert m.switched_at is not None
    if min_pw == 0:
        assert any(s[0] == "tf32x3" for s in m.solves)
