"""Standalone 3D FFT (FFTW-backend semantics) on the GPU against the golden round trips and numpy."""
import os

import numpy as np
import pytest

from oracle import fft as offt

pytestmark = pytest.mark.gpu


def test_golden_roundtrips(dz):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "fft_roundtrip.npz"))
    for key in ("r6", "r234", "r8", "r24"):
        dims = tuple(int(v) for v in d["dims_" + key])
        x = d[key].copy()
        p = dz.Fft3dPlan(*dims)
        y = x.copy()
        p.forward(y)
        p.inverse(y)
        assert np.abs(y - x).max() < float(d["tol"])
        p.close()


# the configs' boxes: Si2 20^3, Al4 27^3, SiGe8 32^3 and 36^3, Si64 75^3, Si216 108^3; plus odd shapes
@pytest.mark.parametrize("dims", [(20, 20, 20), (27, 27, 27), (32, 32, 32), (36, 36, 36), (36, 32, 32), (75, 75, 75),
                                  (108, 108, 108), (75, 12, 10), (4, 5, 6), (1, 8, 3)])
def test_forward_inverse_match_oracle(dz, dims):
    rng = np.random.default_rng(1)
    n = int(np.prod(dims))
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    p = dz.Fft3dPlan(*dims)
    f = x.copy()
    p.forward(f)
    ref = offt.fft3d_forward(x, *dims)
    assert np.abs(f - ref).max() < 1e-12 * np.abs(ref).max()
    g = x.copy()
    p.inverse(g)
    ref2 = offt.fft3d_inverse(x, *dims)
    assert np.abs(g - ref2).max() < 1e-12 * np.abs(ref2).max()
    p.close()
