"""The library's complex GEMMs (dftcuda_complex_gemm) against a torch complex128 product.

Layouts follow the library's own call sites: the Rayleigh-Ritz Gram matrix V^H W (K-contiguous
operands, conjugated A), the subspace rotation V C (one operand K-contiguous, one not), the
projector contraction and its back-projection, and the plain form; both output orientations, so
the tensor-core path runs each product as given and as its transpose.  Shapes include partial
tiles in every dimension and split-K."""
import math

import pytest
import torch

pytestmark = pytest.mark.gpu

# (name, a K-contiguous, b K-contiguous, conj_a, conj_b)
LAYOUTS = [
    ("gram", True, True, True, False),
    ("rotation", True, False, False, False),
    ("projection", True, True, False, False),
    ("backprojection", False, False, False, True),
    ("plain", False, False, False, False),
]

# (M, N, K): both dimensions >= 128 (wide 128 x 256 tiles), partial tiles, split-K, and narrow shapes
SHAPES = [
    (300, 520, 1000),
    (256, 384, 6000),
    (1344, 448, 2000),
    (129, 130, 77),
    (64, 32, 3000),
    (40, 700, 900),
]

# max |error| <= TOL * sqrt(K) * rms(a) * rms(b).  TF32: operand rounding to 10-bit mantissas.
# TF32X3: the tensor cores' FP32 accumulation is not round-to-nearest and its error grows with the
# number of accumulations; the kernels drain it to FP64 every 2048 terms, which holds the error near
# 1e-5 of the largest entry (about 4e-5 of this scale) whatever K is.
TOL = {0: 1e-13, 2: 4e-3, 3: 2e-4}


def _operand(rows, k, kc, gen):
    x = torch.randn(rows, k, dtype=torch.complex128, generator=gen).cuda()
    return x if kc else x.T.contiguous().T  # same values, unit stride along rows


def _case(dz, M, N, K, layout, precision, out_rowmajor, seed):
    _, akc, bkc, cja, cjb = layout
    gen = torch.Generator().manual_seed(seed)
    a = _operand(M, K, akc, gen)
    b = _operand(N, K, bkc, gen)
    o0 = torch.randn(M, N, dtype=torch.complex128, generator=gen).cuda()
    out = o0.clone() if out_rowmajor else o0.T.contiguous().T
    alpha, beta = 0.75, -0.5
    dz.complex_gemm(a, b, out, conj_a=cja, conj_b=cjb, precision=precision, alpha=alpha, beta=beta)
    ref = alpha * ((a.conj() if cja else a) @ (b.conj() if cjb else b).T) + beta * o0
    scale = math.sqrt(K) * a.abs().pow(2).mean().sqrt().item() * b.abs().pow(2).mean().sqrt().item()
    err = (out - ref).abs().max().item()
    return err, scale


@pytest.mark.parametrize("precision", [0, 2, 3], ids=["fp64", "tf32", "tf32x3"])
@pytest.mark.parametrize("layout", LAYOUTS, ids=[l[0] for l in LAYOUTS])
def test_complex_gemm_matches_torch(dz, layout, precision):
    worst = 0.0
    for i, (M, N, K) in enumerate(SHAPES):
        for rowmajor in (False, True):
            err, scale = _case(dz, M, N, K, layout, precision, rowmajor, 100 * i + int(rowmajor))
            assert err <= TOL[precision] * scale, (M, N, K, rowmajor, err / scale)
            worst = max(worst, err / scale)
    # the tensor-core products are genuinely reduced precision, not an FP64 fallback
    if precision == 2:
        assert worst > 1e-8


def test_complex_gemm_tf32x3_is_more_accurate_than_tf32(dz):
    e2, s = _case(dz, 512, 512, 4096, LAYOUTS[0], 2, False, 7)
    e3, _ = _case(dz, 512, 512, 4096, LAYOUTS[0], 3, False, 7)
    assert e3 < e2 / 10, (e2 / s, e3 / s)


def test_complex_gemm_tf32x3_error_does_not_grow_with_k(dz):
    """Gram-shaped products with K from 2e3 to 1.2e5: the FP64 drains keep the error flat."""
    errs = []
    for K in (2048, 120000):
        gen = torch.Generator().manual_seed(K)
        a = (torch.randn(256, K, dtype=torch.complex128, generator=gen) / math.sqrt(K)).cuda()
        b = (torch.randn(256, K, dtype=torch.complex128, generator=gen) / math.sqrt(K)).cuda()
        ref = a.conj() @ b.T
        out = dz.complex_gemm(a, b, conj_a=True, precision=3)
        errs.append((out - ref).abs().max().item() / ref.abs().max().item())
    assert errs[1] < 4 * errs[0] + 1e-6, errs
    assert errs[1] < 1e-4, errs


def test_complex_gemm_rejects_fp32_and_bad_shapes(dz):
    a = torch.zeros(8, 8, dtype=torch.complex128, device="cuda")
    with pytest.raises(dz.DftCudaError):
        dz.complex_gemm(a, a, precision=dz.PRECISION_FP32)
    with pytest.raises(dz.DftCudaError):
        dz.complex_gemm(a, torch.zeros(8, 9, dtype=torch.complex128, device="cuda"))
