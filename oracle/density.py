"""Band-density accumulation, occupations and Fermi level (oracle; test infrastructure only).

Restates:
  src/features/scf/kpoint/density.zig:90-143   accumulate_band_contributions (fixed occupations:
                                                occ = 1 except the last occupied band, occ = N_e/2 - (nocc-1);
                                                weight = w_k * occ * 2)
  src/features/scf/kpoint/density.zig:444-474  accumulate_band_density_fft (scatter into the centred grid,
                                                mapped inverse FFT with xN, rho += weight |psi|^2 / Omega)
  src/features/scf/kpoint/density.zig:381-417  accumulate_smearing_band (FD occupation, entropy)
  src/features/scf/fermi_level.zig:7-124       smearing_occ, smearing_entropy, find_fermi_level
"""
from __future__ import annotations

import math

import numpy as np

from . import fft as offt
from .pw import Grid, PwGridMap, build_fft_index_map


def band_density(grid: Grid, pwmap: PwGridMap, coeffs: np.ndarray, weight: float, inv_volume: float) -> np.ndarray:
    """One band's contribution weight*|psi(r)|^2/Omega on the FFT-order grid (density.zig:444-474)."""
    total = grid.count
    recip = np.zeros(total, dtype=np.complex128)
    pwmap.scatter(coeffs, recip)
    idx_map = build_fft_index_map(grid)
    work = recip[idx_map] * float(total)
    psi = offt.fft3d_inverse(work, grid.nx, grid.ny, grid.nz)
    dens = (psi.real * psi.real + psi.imag * psi.imag) * inv_volume
    return weight * dens


def fixed_occupations(nelec: float, nocc: int, nbands: int):
    """density.zig:98-106."""
    occ_last = 0.0 if nocc == 0 else nelec / 2.0 - float(nocc - 1)
    occ = np.zeros(nbands)
    for b in range(min(nocc, nbands)):
        occ[b] = occ_last if b + 1 == nocc else 1.0
    return occ


def accumulate_density(grid: Grid, pwmap: PwGridMap, vectors: np.ndarray, weights: np.ndarray, inv_volume: float):
    """rho(r) = sum_b weights_b |psi_b(r)|^2 / Omega, bands with weight <= 0 skipped (density.zig:104-107,386-388)."""
    rho = np.zeros(grid.count)
    for b in range(vectors.shape[0]):
        if weights[b] <= 0.0:
            continue
        rho += band_density(grid, pwmap, vectors[b], float(weights[b]), inv_volume)
    return rho


def smearing_occ(energy: float, mu: float, sigma: float, method: str = "fermi_dirac") -> float:
    """fermi_level.zig:7-11."""
    if sigma <= 0.0 or method == "none":
        return 1.0 if energy <= mu else 0.0
    return 1.0 / (1.0 + math.exp((energy - mu) / sigma))


def smearing_entropy(occ: float) -> float:
    """fermi_level.zig:15-19."""
    eps = 1e-12
    if occ <= eps or occ >= 1.0 - eps:
        return 0.0
    return -(occ * math.log(occ) + (1.0 - occ) * math.log(1.0 - occ))


def electron_count(mu, sigma, kweights, values, spin_factor=2.0, method="fermi_dirac"):
    count = 0.0
    for wk, vals in zip(kweights, values):
        weight = spin_factor * wk
        for e in vals:
            count += weight * smearing_occ(float(e), mu, sigma, method)
    return count


def find_fermi_level(nelec, sigma, kweights, values, spin_factor=2.0, method="fermi_dirac") -> float:
    """fermi_level.zig:61-124: bracket with padding max(10 sigma, 1e-3) (<= 12 doublings),
    then <= 80 bisections stopping at |N(mu) - N_e| < 1e-8."""
    allv = np.concatenate([np.asarray(v, dtype=np.float64) for v in values])
    lo_e, hi_e = float(allv.min()), float(allv.max())
    pad = max(10.0 * sigma, 1e-3)
    low, high = lo_e - pad, hi_e + pad
    cl = electron_count(low, sigma, kweights, values, spin_factor, method)
    ch = electron_count(high, sigma, kweights, values, spin_factor, method)
    expand = 0
    while (cl > nelec or ch < nelec) and expand < 12:
        pad *= 2.0
        low, high = lo_e - pad, hi_e + pad
        cl = electron_count(low, sigma, kweights, values, spin_factor, method)
        ch = electron_count(high, sigma, kweights, values, spin_factor, method)
        expand += 1
    left, right = low, high
    for _ in range(80):
        mid = 0.5 * (left + right)
        c = electron_count(mid, sigma, kweights, values, spin_factor, method)
        if abs(c - nelec) < 1e-8:
            return mid
        if c > nelec:
            right = mid
        else:
            left = mid
    return 0.5 * (left + right)
