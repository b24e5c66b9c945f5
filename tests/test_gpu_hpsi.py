"""H|psi> on the GPU (through the C ABI) against the oracle's restatement of apply.zig.

Tolerances: FP64 path max relative error 1e-11 (FFT round-off only); FP32 FFT passes 5e-5."""
import numpy as np
import pytest

from oracle import fft as offt
from tests.helpers import kproblem, make_context, random_block, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    ("si2", 20.0, (0.25, 0.125, 0.0)),
    ("si2", 20.0, (0.0, 0.0, 0.0)),
    ("al4", 25.0, (0.1, 0.2, 0.3)),
    ("sige8", 20.0, (0.25, 0.25, 0.25)),
    ("si8", 20.0, (0.5, 0.0, 0.0)),
]


@pytest.mark.parametrize("name,ecut,k", CASES)
def test_apply_batched_fp64(dz, name, ecut, k):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 7, 11)
    y = kc.apply_hamiltonian_batched(x)
    ref = kp.ctx.apply_batch(x)
    assert rel_err(y, ref) < 1e-11
    # single-column Operator.apply agrees with the batch
    y1 = kc.apply_hamiltonian(x[3])
    assert rel_err(y1, ref[3]) < 1e-11
    kc.close()


def test_apply_batched_si64_full_box(dz):
    """Si64 2x2x2 supercell, 30 Ry, 75^3 box, 64 atoms of projectors; 36 columns span two
    box-workspace chunks."""
    kp = kproblem("si64", 30.0)
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 36, 5)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-11
    kc.close()


def test_apply_many_columns_chunked(dz):
    """More columns than one box-workspace chunk holds."""
    kp = kproblem("si8", 20.0)
    kc = make_context(dz, kp)
    kc_budget_cols = 70
    x = random_block(kp.ctx.n, kc_budget_cols, 2)
    y = kc.apply_hamiltonian_batched(x)
    ref = kp.ctx.apply_batch(x)
    assert rel_err(y, ref) < 1e-11
    kc.close()


def test_host_pipeline_uneven_chunks(dz):
    """From 256 host columns the copies run in 64-column end chunks around larger middle chunks
    (here 64, 128, 44, 64): every column equals the device-pointer path, the end chunks the oracle."""
    import torch

    kp = kproblem("si8", 20.0)
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 300, 4)
    y = kc.apply_hamiltonian_batched(x)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    kc.apply_hamiltonian_batched(xd, yd, kp.ctx.n, 300)
    assert rel_err(y, yd.cpu().numpy()) < 1e-13
    for cols in (slice(0, 6), slice(190, 196), slice(294, 300)):
        assert rel_err(y[cols], kp.ctx.apply_batch(x[cols])) < 1e-11
    kc.close()


@pytest.mark.parametrize("name,ecut,k", CASES[:3])
def test_apply_batched_fp32_passes(dz, name, ecut, k):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp, precision=dz.PRECISION_FP32)
    x = random_block(kp.ctx.n, 5, 3)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 5e-5
    kc.close()


def test_device_pointer_path_matches_host(dz):
    import torch

    kp = kproblem("si2", 20.0, (0.25, 0.0, 0.0))
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 4, 9)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    kc.apply_hamiltonian_batched(xd, yd, kp.ctx.n, 4)
    assert rel_err(yd.cpu().numpy(), kc.apply_hamiltonian_batched(x)) < 1e-14
    kc.close()


def test_nonlocal_energies(dz):
    kp = kproblem("si8", 20.0, (0.25, 0.0, 0.0))
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 4, 4)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    e = kc.nonlocal_energies(x)
    ref = np.array([kp.ctx.nonlocal_energy(v) for v in x])
    assert np.abs(e - ref).max() < 1e-11 * max(1.0, np.abs(ref).max())
    kc.close()


def test_local_potential_kat_through_abi(dz):
    """src/tests.zig:872-973 on the full 4^3 box through the C ABI: V psi = V_G for psi = delta(G=0)."""
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "local_potential_kat.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    N = nx * ny * nz
    # the full box as a basis, in FFT order: Miller index of position i is index_to_freq
    def freq(i, n):
        return i if i <= (n - 1) // 2 else i - n

    hkl = np.array([[freq(x, nx), freq(y, ny), freq(z, nz)] for z in range(nz) for y in range(ny) for x in range(nx)], dtype=np.int32)
    kc = dz.KpointContext(nx, ny, nz, 1.0, hkl, np.zeros(N), np.zeros((N, 3)))
    local_r = offt.fft3d_inverse(d["v1"] * N, nx, ny, nz).real.copy()
    kc.set_vloc(local_r)
    out = kc.apply_hamiltonian(d["psi1"])
    assert np.abs(out[:5] - d["expected1"][:5]).max() < float(d["tol"])
    assert np.abs(out - d["expected1"]).max() < float(d["tol"])
    kc.close()


def test_local_potential_kat2_through_abi(dz):
    """src/tests.zig:975-1104 through the C ABI: with V(r) = N IFFT(V_G) for V_G = 1 at G = 0 and 0.5 at
    G = (+-1, 0, 0), H psi for psi = delta(G=0) equals the direct O(N^2) convolution of V_G and psi
    (expected2 of the fixture) to the reference's 1e-10."""
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "local_potential_kat.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    N = nx * ny * nz

    def freq(i, n):
        return i if i <= (n - 1) // 2 else i - n

    hkl = np.array([[freq(x, nx), freq(y, ny), freq(z, nz)] for z in range(nz) for y in range(ny) for x in range(nx)], dtype=np.int32)
    kc = dz.KpointContext(nx, ny, nz, 1.0, hkl, np.zeros(N), np.zeros((N, 3)))
    kc.set_vloc(offt.fft3d_inverse(d["v2"] * N, nx, ny, nz).real.copy())
    out = kc.apply_hamiltonian(d["psi2"])
    assert np.abs(out - d["expected2"]).max() < float(d["tol"])
    kc.close()


def test_errors_map_to_reference(dz):
    kp = kproblem("si2", 20.0)
    kc = make_context(dz, kp)
    with pytest.raises(dz.InvalidMatrixSize):
        kc.apply_hamiltonian_batched(np.zeros((2, kp.ctx.n + 1), np.complex128), n=kp.ctx.n + 1, ncols=2)
    kc.close()
    b = kp.ctx.basis
    with pytest.raises(dz.InvalidGrid):
        dz.KpointContext(6, 6, 6, kp.grid.volume, b.hkl, b.kinetic, b.cart)
    with pytest.raises(dz.Unsupported):
        dz.KpointContext(21, 20, 20, kp.grid.volume, b.hkl, b.kinetic, b.cart)


def test_zero_columns_is_a_noop(dz):
    kp = kproblem("si2", 20.0)
    kc = make_context(dz, kp)
    y = kc.apply_hamiltonian_batched(np.zeros((0, kp.ctx.n), np.complex128), ncols=0)
    assert y.shape == (0, kp.ctx.n)
    kc.close()


@pytest.mark.parametrize("path", ["generic", "planes", "sticks"])
@pytest.mark.parametrize("name,ecut,k,prec", [("si2", 20.0, (0.25, 0.125, 0.0), 0), ("sige8", 20.0, (0.25, 0.25, 0.25), 0),
                                              ("al4", 25.0, (0.1, 0.2, 0.3), 1), ("si8", 20.0, (0.5, 0.0, 0.0), 1)])
def test_all_fft_paths_match_oracle(dz, monkeypatch, path, name, ecut, k, prec):
    """The three local-operator paths give the oracle's H|psi> and density: the stick-layout passes
    (DFTCUDA_LOCAL=sticks, where nx = ny; the default from 96 points along x), the four-step
    plane-layout passes (DFTCUDA_LOCAL=planes, the default below) and the stage-by-stage passes
    (DFTCUDA_FFT_PATH=generic).  The profile reports the layout that ran."""
    from oracle import density as odens

    monkeypatch.delenv("DFTCUDA_FFT_PATH", raising=False)
    monkeypatch.delenv("DFTCUDA_LOCAL", raising=False)
    if path == "generic":
        monkeypatch.setenv("DFTCUDA_FFT_PATH", "generic")
    elif path == "planes":
        monkeypatch.setenv("DFTCUDA_LOCAL", "planes")
    else:
        monkeypatch.setenv("DFTCUDA_LOCAL", "sticks")
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp, precision=prec)
    x = random_block(kp.ctx.n, 6, 21)
    tol = 1e-11 if prec == 0 else 5e-5
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < tol
    layout = kc.profile()["local_layout"]
    if path == "generic":
        assert layout == 0
    elif path == "planes":
        assert layout == 1
    elif kp.grid.nx == kp.grid.ny:
        assert layout == 2
    w = np.array([2.0, 1.0, 0.5, 0.25, 0.0, 1.5])
    rho = np.zeros(kp.grid.count)
    kc.accumulate_band_density(x, w, rho)
    ref = odens.accumulate_density(kp.grid, kp.ctx.map, x, w, 1.0 / kp.grid.volume)
    assert rel_err(rho, ref) < (1e-12 if prec == 0 else 5e-5)
    kc.close()


def test_autotune_keeps_results(dz):
    """The autotuner times launch configurations on the context's own data; whatever it picks, H|psi>
    still matches the oracle at the FP64 bar."""
    kp = kproblem("si8", 20.0, (0.25, 0.0, 0.0))
    kc = make_context(dz, kp)
    rep = kc.autotune(48)
    assert rep["candidates"] >= 4 and rep["tuned_ms"] <= rep["default_ms"] + 1e-9
    assert rep["fft_path"] in (0, 1, 2) and rep["box_budget_mb"] > 0
    x = random_block(kp.ctx.n, 48, 5)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-11
    kc.close()


@pytest.mark.parametrize("name,ecut,k", [("si8", 15.0, (0.25, 0.0, 0.125)), ("al4", 15.0, (0.1, 0.2, 0.3))])
def test_hamiltonian_is_hermitian(dz, name, ecut, k):
    """The reference's Hamiltonian Hermiticity test (src/tests.zig:765-831) on the device operator:
    <x|H y> = <H x|y> for random blocks, local and nonlocal parts included, to FP64 rounding."""
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 4, 3)
    y = random_block(kp.ctx.n, 4, 4)
    hx = kc.apply_hamiltonian_batched(x)
    hy = kc.apply_hamiltonian_batched(y)
    a = x.conj() @ hy.T
    b = hx.conj() @ y.T
    assert np.abs(a - b).max() < 1e-12 * np.abs(a).max()
    kc.close()


def test_apply_equals_dense_hamiltonian(dz):
    """The dense-versus-apply check of the reference (apply.zig:660-729): the device operator applied
    to every unit vector reproduces the oracle's dense H (Si2, 20 Ry, off-Gamma) column by column."""
    kp = kproblem("si2", 20.0, (0.25, 0.125, 0.0))
    kc = make_context(dz, kp)
    n = kp.ctx.n
    eye = np.eye(n, dtype=np.complex128)
    h = kc.apply_hamiltonian_batched(eye)  # row b = H e_b = column b of H
    dense = kp.ctx.dense_hamiltonian()
    assert np.abs(h.T - dense).max() < 1e-11 * np.abs(dense).max()
    kc.close()
