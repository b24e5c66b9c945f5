"""Internal consistency of the oracle on the synthetic cells (CPU only)."""
import numpy as np

from oracle import density as odens
from oracle import lobpcg
from tests.helpers import kproblem, random_block


def test_hamiltonian_hermitian_and_batched_equals_scalar():
    kp = kproblem("si2", 12.0, (0.25, 0.0, 0.0))
    h = kp.ctx.dense_hamiltonian()
    assert np.abs(h - h.conj().T).max() < 1e-13
    x = random_block(kp.ctx.n, 3, 7)
    yb = kp.ctx.apply_batch(x)
    ys = np.array([kp.ctx.apply(c) for c in x])
    assert np.abs(yb - ys).max() < 1e-12 * np.abs(ys).max()


def test_davidson_matches_dense():
    kp = kproblem("si2", 12.0, (0.125, 0.25, 0.0))
    h = kp.ctx.dense_hamiltonian()
    ev = np.linalg.eigvalsh(h)[:8]
    r = lobpcg.solve(lobpcg.Operator(kp.ctx.n, kp.ctx.apply_batch), kp.ctx.basis.kinetic, 8, lobpcg.Options(max_iter=200, tol=1e-9))
    assert r.converged
    assert np.abs(r.values - ev).max() < 1e-9


def test_density_integrates_to_weight():
    kp = kproblem("si2", 12.0)
    rng = np.random.default_rng(0)
    n = kp.ctx.n
    v = random_block(n, 3, 1)
    q, _ = np.linalg.qr(v.T)
    vec = q.T
    w = np.array([2.0, 1.5, 0.5])
    rho = odens.accumulate_density(kp.grid, kp.ctx.map, vec, w, 1.0 / kp.grid.volume)
    # sum_r rho dV = sum_b w_b <psi_b|psi_b> with the reference's normalisation (plane-wave sum)
    total = rho.sum() * kp.grid.volume / kp.grid.count
    assert abs(total - w.sum()) < 1e-10


def test_fermi_level_bisection():
    vals = [np.array([-0.5, 0.1, 0.2, 0.3]), np.array([-0.4, 0.15, 0.25, 0.5])]
    w = [0.5, 0.5]
    mu = odens.find_fermi_level(4.0, 0.01, w, vals)
    n = odens.electron_count(mu, 0.01, w, vals)
    assert abs(n - 4.0) < 1e-7
