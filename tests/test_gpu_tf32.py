"""TF32 mode: FP32 FFT passes and tcgen05 tensor-core projector GEMMs, against the FP64 oracle.

TF32 keeps 10 mantissa bits, so the nonlocal term carries a relative error of order 1e-3 of its own
size; the tests bound it at 4e-3 of the largest |V_nl psi| entry and the whole H psi at 2e-3."""
import numpy as np
import pytest

from tests.helpers import kproblem, make_context, random_block, rel_err

pytestmark = pytest.mark.gpu


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
