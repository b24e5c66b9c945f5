"""3D complex FFT with dft-zig's FFTW-backend semantics (oracle; test infrastructure only).

Restates src/lib/fft/fftw_fft.zig:91-166: ``fftw_plan_dft_3d(nz, ny, nx)`` on a
buffer indexed ``x + nx*(y + ny*z)`` (x fastest); forward is FFTW_FORWARD
(e^{-i}), unnormalised; inverse is FFTW_BACKWARD (e^{+i}) followed by a 1/N
scale in the wrapper.  numpy's pocketfft computes the same DFT definitions.
"""
from __future__ import annotations

import numpy as np


def fft3d_forward(data: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    a = np.asarray(data, dtype=np.complex128).reshape(nz, ny, nx)
    return np.fft.fftn(a, axes=(0, 1, 2)).ravel()


def fft3d_inverse(data: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    a = np.asarray(data, dtype=np.complex128).reshape(nz, ny, nx)
    return np.fft.ifftn(a, axes=(0, 1, 2)).ravel()


def dft3d_direct(data: np.ndarray, nx: int, ny: int, nz: int, sign: int) -> np.ndarray:
    """O(N^2) direct DFT used to pin the FFT on tiny boxes (the reference's radix tests
    compare against a direct DFT the same way: src/lib/fft/mixed_radix.zig:862-1262)."""
    a = np.asarray(data, dtype=np.complex128).reshape(nz, ny, nx)
    out = a
    for axis, n in ((2, nx), (1, ny), (0, nz)):
        j = np.arange(n)
        w = np.exp(sign * 2j * np.pi * np.outer(j, j) / n)
        out = np.moveaxis(np.tensordot(w, np.moveaxis(out, axis, 0), axes=(1, 0)), 0, axis)
    return out.ravel()
