"""Failure paths on the GPU, tested without faulting, trapping or hanging the device.

Every device-side wait in the library is bounded.  dftcuda_debug_set_wait_limits makes the subspace
eigensolver's grid barrier wait for an arrival that no block makes, with a short poll budget, so the
wait runs out: the blocks set the error flag and return, the call reports DFTCUDA_ERR_TIMEOUT, and a
normal call afterwards (on the same context) must succeed.  A NaN injected on the host into one
column of psi must come back as a clean status with the NaN confined to that column.
dftcuda_debug_fail_alloc makes one device allocation fail as cudaMalloc does on a full device: the
call reports DFTCUDA_ERR_OUT_OF_MEMORY and the context stays usable.
"""
import numpy as np
import pytest

from tests.helpers import kproblem, make_context, random_block, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture
def limits(dz):
    yield dz.debug_set_wait_limits
    dz.debug_set_wait_limits()  # defaults again, whatever the test did


def _hermitian(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return a + a.conj().T


def test_grid_barrier_timeout_reports_and_recovers(dz, limits):
    a = _hermitian(200, 1)  # 200 >= 96: the tridiagonal solver with its cooperative grid barrier
    limits(4096, True)
    with pytest.raises(dz.Timeout):
        dz.hermitian_eigen_decomp(a, 20)
    limits()
    r = dz.hermitian_eigen_decomp(a, 20)
    ref = np.linalg.eigvalsh(a)[:20]
    assert np.abs(r.values - ref).max() < 1e-10 * np.abs(ref).max()


def test_eigensolver_timeout_leaves_context_usable(dz, limits):
    kp = kproblem("si8", 20.0, (0.25, 0.0, 0.0))
    kc = make_context(dz, kp)
    limits(4096, True)
    with pytest.raises(dz.Timeout):  # 100 bands: the first Rayleigh-Ritz step is 100 x 100
        kc.hermitian_eigen_decomp_iterative(kp.ctx.basis.kinetic, 100, dz.Options(max_iter=3, tol=1e-6))
    limits()
    r = kc.hermitian_eigen_decomp_iterative(kp.ctx.basis.kinetic, 100, dz.Options(max_iter=3, tol=1e-6))
    assert np.isfinite(r.values).all()
    x = random_block(kp.ctx.n, 3, 8)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-11
    kc.close()


def test_nan_in_one_column_is_confined(dz):
    kp = kproblem("si2", 20.0, (0.25, 0.125, 0.0))
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 5, 9)
    bad = x.copy()
    bad[2, 17] = np.nan
    y = kc.apply_hamiltonian_batched(bad)  # a clean status: no exception
    assert not np.isfinite(y[2]).all()
    keep = [0, 1, 3, 4]
    assert rel_err(y[keep], kp.ctx.apply_batch(x[keep])) < 1e-11
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-11  # the context is unharmed
    kc.close()


@pytest.fixture
def fail_alloc(dz):
    yield dz.debug_fail_alloc
    dz.debug_fail_alloc()  # cancel whatever the test planned


@pytest.mark.parametrize("after", [0, 1, 2])
def test_allocation_failure_reports_and_recovers(dz, fail_alloc, after):
    """The after-th device allocation of the first H|psi> call and of the first Davidson solve on a
    fresh context fails: each call raises OutOfMemory, then succeeds on the same context."""
    kp = kproblem("si8", 20.0, (0.25, 0.0, 0.0))
    kc = make_context(dz, kp)
    x = random_block(kp.ctx.n, 6, 4)
    fail_alloc(after)
    with pytest.raises(dz.OutOfMemory):
        kc.apply_hamiltonian_batched(x)
    fail_alloc()
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-11
    opts = dz.Options(max_iter=3, tol=1e-6)
    fail_alloc(after)
    with pytest.raises(dz.OutOfMemory):
        kc.hermitian_eigen_decomp_iterative(kp.ctx.basis.kinetic, 20, opts)
    fail_alloc()
    r = kc.hermitian_eigen_decomp_iterative(kp.ctx.basis.kinetic, 20, opts)
    assert np.isfinite(r.values).all()
    x2 = random_block(kp.ctx.n, 3, 5)
    assert rel_err(kc.apply_hamiltonian_batched(x2), kp.ctx.apply_batch(x2)) < 1e-11
    kc.close()
