"""Dense Hermitian eigensolver (Householder tridiagonalisation + multisection + inverse iteration +
back-transformation) against LAPACK (numpy.linalg.eigh), and inside the Davidson loop against the
one-CTA Jacobi path.

Bars: eigenvalues within 1e-12 ||A||, residual ||A v - lambda v|| within 1e-12 ||A||, eigenvectors
orthonormal to 1e-10 (the Rayleigh-Ritz step only needs the spanned subspace, so phases are free)."""
import os

import numpy as np
import pytest

from tests.helpers import kproblem, make_context

pytestmark = pytest.mark.gpu


def _rand_herm(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return scale * (x + x.conj().T) / 2


def _check(a, r, nev):
    ref = np.linalg.eigvalsh(a)[:nev]
    an = max(1.0, np.abs(ref).max(), np.linalg.norm(a, 2))
    v = r.vectors  # (nev, n)
    assert r.values.shape == (nev,) and v.shape == (nev, a.shape[0])
    assert np.all(np.diff(r.values) >= -1e-12 * an)
    assert np.abs(r.values - ref).max() < 1e-12 * an
    res = np.linalg.norm(a @ v.T - v.T * r.values, axis=0)
    assert res.max() < 1e-12 * an * np.sqrt(a.shape[0])
    assert np.abs(v.conj() @ v.T - np.eye(nev)).max() < 1e-10


@pytest.mark.parametrize("n,nev", [(1, 1), (2, 2), (3, 2), (17, 17), (64, 20), (95, 40), (96, 96), (200, 64), (648, 164)])
def test_random_hermitian(dz, n, nev):
    a = _rand_herm(n, seed=n)
    _check(a, dz.hermitian_eigen_decomp(a, nev), nev)


def test_subspace_sized_problem(dz):
    """The Si216 Davidson shape: m = 1800, 448 lowest pairs, spectrum in Ry."""
    a = _rand_herm(1800, seed=7, scale=0.05)
    _check(a, dz.hermitian_eigen_decomp(a, 448), 448)


def test_degenerate_spectrum(dz):
    rng = np.random.default_rng(3)
    n = 90
    q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    d = np.repeat(np.arange(30.0) * 0.1, 3)  # triplets, as at symmetric k-points
    a = q @ np.diag(d) @ q.conj().T
    a = (a + a.conj().T) / 2
    _check(a, dz.hermitian_eigen_decomp(a, 45), 45)


def test_large_eigenvalue_clusters(dz):
    """Groups beyond a warp: 40 equal eigenvalues and 12 within 1e-9 of each other, between spread
    singletons, so the inverse iteration re-orthogonalises long groups."""
    rng = np.random.default_rng(5)
    n = 400
    q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    d = np.sort(np.r_[np.linspace(-3.0, 8.0, n - 52), np.full(40, 0.5), 2.0 + 1e-9 * np.arange(12)])
    a = q @ np.diag(d) @ q.conj().T
    a = (a + a.conj().T) / 2
    _check(a, dz.hermitian_eigen_decomp(a, 240), 240)


def test_diagonal_and_identity(dz):
    a = np.diag(np.r_[np.full(6, 2.0), np.full(5, -1.0), [0.5]]).astype(np.complex128)
    _check(a, dz.hermitian_eigen_decomp(a), 12)
    _check(np.eye(40, dtype=np.complex128), dz.hermitian_eigen_decomp(np.eye(40, dtype=np.complex128), 10), 10)


def test_reads_upper_triangle_only(dz):
    a = _rand_herm(50, seed=11)
    junk = a.copy()
    il = np.tril_indices(50, -1)
    junk[il] = 123.0 + 45.0j
    r1 = dz.hermitian_eigen_decomp(a, 20)
    r2 = dz.hermitian_eigen_decomp(junk, 20)
    assert np.array_equal(r1.values, r2.values)


def test_size_errors(dz):
    with pytest.raises(dz.InvalidMatrixSize):
        dz.hermitian_eigen_decomp(np.eye(4, dtype=np.complex128), 5)


@pytest.mark.parametrize("cell,ecut,nb", [("si8", 15.0, 40), ("al4", 15.0, 24)])
def test_davidson_tridiag_matches_jacobi(dz, cell, ecut, nb):
    """Subspaces of 4 nb + 8 >= 96 columns: the tridiagonal path (default there) and the Jacobi
    path reach the same converged eigenvalues."""
    kp = kproblem(cell, ecut, (0.25, 0.125, 0.0))
    diag = kp.ctx.basis.kinetic
    out = {}
    for mode in ("jacobi", "tridiag"):
        os.environ["DFTCUDA_SUBSPACE_EIG"] = mode
        try:
            kc = make_context(dz, kp)
            out[mode] = kc.hermitian_eigen_decomp_iterative(diag, nb, dz.Options(max_iter=200, tol=1e-9))
            kc.close()
        finally:
            del os.environ["DFTCUDA_SUBSPACE_EIG"]
    assert out["jacobi"].converged and out["tridiag"].converged
    assert np.abs(out["jacobi"].values - out["tridiag"].values).max() < 1e-9
    dense = np.linalg.eigvalsh(kp.ctx.dense_hamiltonian())[:nb]
    assert np.abs(out["tridiag"].values - dense).max() < 1e-7


def test_incremental_gram_matches_full_rebuild(dz):
    """The Rayleigh-Ritz matrix extended by the new columns only (default) and rebuilt in full every
    iteration (the reference's order of work) give the same converged eigenvalues."""
    kp = kproblem("si8", 15.0, (0.0, 0.0, 0.0))
    diag = kp.ctx.basis.kinetic
    out = {}
    for mode in ("full", "incremental"):
        if mode == "full":
            os.environ["DFTCUDA_GRAM"] = "full"
        try:
            kc = make_context(dz, kp)
            out[mode] = kc.hermitian_eigen_decomp_iterative(diag, 32, dz.Options(max_iter=200, tol=1e-9))
            kc.close()
        finally:
            os.environ.pop("DFTCUDA_GRAM", None)
    assert out["full"].converged and out["incremental"].converged
    assert np.abs(out["full"].values - out["incremental"].values).max() < 1e-9
