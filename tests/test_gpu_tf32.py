"""TF32 and TF32X3 modes: FP32 FFT passes and tcgen05 tensor-core GEMMs, against the FP64 oracle.

TF32 keeps 10 mantissa bits, so the nonlocal term carries a relative error of order 1e-3 of its own
size; the tests bound it at 4e-3 of the largest |V_nl psi| entry and the whole H psi at 2e-3.

These cases are small enough that a TF32 context would hand its contractions to the FP64 GEMM
(below 5e8 useful FLOPs); DFTCUDA_TC_MIN_FLOP=0 keeps every one of them on the tensor cores here.
test_small_contractions_take_fp64 checks the default: FP64-exact results in a TF32 context."""
import numpy as np
import pytest

from tests.helpers import kproblem, make_context, random_block, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _tensor_cores_for_every_size(monkeypatch, request):
    if request.node.name.startswith("test_small_contractions_take_fp64"):
        monkeypatch.delenv("DFTCUDA_TC_MIN_FLOP", raising=False)
    else:
        monkeypatch.setenv("DFTCUDA_TC_MIN_FLOP", "0")


def test_small_contractions_take_fp64(dz):
    """With the default threshold a TF32 context's projector GEMMs on Si2 (a few MFLOP) run on the
    FP64 GEMM: the nonlocal term then matches the oracle at the FP64 bar, not the TF32 one."""
    kp = kproblem("si2", 20.0, (0.25, 0.125, 0.0))
    kc = make_context(dz, kp, precision=dz.PRECISION_TF32)
    kc.set_vloc(np.zeros(kp.grid.count))  # the FP32 FFT passes then add exactly zero
    x = random_block(kp.ctx.n, 5, 3)
    y = kc.apply_hamiltonian_batched(x) - x * kp.ctx.basis.kinetic[None, :]
    ref = kp.ctx.apply_nonlocal_batched(x)
    assert np.abs(y - ref).max() < 1e-11 * np.abs(ref).max()
    kc.close()


@pytest.mark.parametrize("name,ecut,k,ncols", [("si2", 20.0, (0.25, 0.125, 0.0), 5), ("si8", 20.0, (0.5, 0.0, 0.0), 70), ("sige8", 20.0, (0.25, 0.25, 0.25), 9)])
def test_tf32_nonlocal_matches_oracle(dz, name, ecut, k, ncols):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp, precision=dz.PRECISION_TF32)
    kc.set_vloc(np.zeros(kp.grid.count))
    x = random_block(kp.ctx.n, ncols, 31)
    y = kc.apply_hamiltonian_batched(x) - x * kp.ctx.basis.kinetic[None, :]
    ref = kp.ctx.apply_nonlocal_batched(x)
    assert np.abs(y - ref).max() < 4e-3 * np.abs(ref).max()
    kc.close()


def test_tf32_full_h_matches_oracle(dz):
    kp = kproblem("si64", 30.0)
    kc = make_context(dz, kp, precision=dz.PRECISION_TF32)
    x = random_block(kp.ctx.n, 40, 7)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 2e-3
    kc.close()


# ---- TF32X3: split hi + lo operands, three MMAs per real product ----------------------------------
# Representation error 2^-22 per operand and FP32 accumulation: ~1e-6 of |V_nl psi|.


@pytest.mark.parametrize("name,ecut,k,ncols", [("si2", 20.0, (0.25, 0.125, 0.0), 5), ("si8", 20.0, (0.5, 0.0, 0.0), 70), ("sige8", 20.0, (0.25, 0.25, 0.25), 9)])
def test_tf32x3_nonlocal_matches_oracle(dz, name, ecut, k, ncols):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp, precision=dz.PRECISION_TF32X3)
    kc.set_vloc(np.zeros(kp.grid.count))
    x = random_block(kp.ctx.n, ncols, 31)
    y = kc.apply_hamiltonian_batched(x) - x * kp.ctx.basis.kinetic[None, :]
    ref = kp.ctx.apply_nonlocal_batched(x)
    assert np.abs(y - ref).max() < 1e-5 * np.abs(ref).max()
    kc.close()


def test_tf32x3_full_h_matches_oracle(dz):
    kp = kproblem("si64", 30.0)
    kc = make_context(dz, kp, precision=dz.PRECISION_TF32X3)
    x = random_block(kp.ctx.n, 40, 7)
    assert rel_err(kc.apply_hamiltonian_batched(x), kp.ctx.apply_batch(x)) < 1e-5
    kc.close()


def test_tf32x3_davidson_eigenvalues(dz):
    """Davidson in a TF32X3 context (FP32 FFTs, split-TF32 projector and Rayleigh-Ritz GEMMs, FP64
    orthonormalisation and subspace eigensolver): eigenvalues within 5e-5 Ry of the FP64 solve.
    The bound is the FP32 floor of H|psi>: relative error ~1e-6 of ||H|| (kinetic up to the 15 Ry
    cutoff plus the potential), i.e. a few 1e-5 Ry; the FP64 switch near convergence removes it."""
    kp = kproblem("si8", 15.0, (0.25, 0.0, 0.0))
    diag = kp.ctx.basis.kinetic
    vals = {}
    for prec in (dz.PRECISION_FP64, dz.PRECISION_TF32X3):
        kc = make_context(dz, kp, precision=prec)
        r = kc.hermitian_eigen_decomp_iterative(diag, 24, dz.Options(max_iter=100, tol=1e-4))
        vals[prec] = r.values
        kc.close()
    assert np.abs(vals[dz.PRECISION_FP64] - vals[dz.PRECISION_TF32X3]).max() < 5e-5
