"""Test infrastructure: the CPU restatement of the reference's density symmetrisation, which the
device entry point dftcuda_symmetrize_density is checked against, and of the space-group search
that produces its inputs (the search stays with the caller; tests use it to make operations).
Only tests use this module.

  symmetrize_density  src/features/scf/density_symmetry.zig:27-94
  symmetry_ops        src/features/symmetry/symmetry.zig:150-330 (build_symmetry_ops,
                      try_append_rotation, lattice_symmetric, find_translations,
                      translation_valid); SymOp.k_rot = (rot^-1)^T (symmetry.zig:229-233)
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from oracle import potential as op


def _wrap01(v):
    v = np.asarray(v, dtype=np.float64)
    return v - np.floor(v)


def _frac_close(a, b, tol):
    d = _wrap01(np.asarray(a) - np.asarray(b))
    d = np.minimum(d, 1.0 - d)
    return bool(np.all(d < tol))


def symmetry_ops(cell, frac_positions, species, tol=1e-5):
    """Integer rotations with entries in {-1, 0, 1} (in lattice coordinates), det +-1, that keep the
    lattice metric, each with every fractional translation that maps the atoms onto atoms of the
    same species; returns a list of (rot, k_rot, trans), k_rot = (rot^-1)^T acting on Miller
    indices.  The search order follows build_symmetry_ops."""
    cell = np.asarray(cell, dtype=np.float64)
    metric = cell @ cell.T
    frac = _wrap01(frac_positions)
    species = list(species)
    ops = []
    for m in itertools.product((-1, 0, 1), repeat=9):
        rot = np.array(m, dtype=np.int64).reshape(3, 3)
        det = int(round(np.linalg.det(rot)))
        if det not in (1, -1):
            continue
        if np.abs(rot.T @ metric @ rot - metric).max() > tol:  # lattice_symmetric
            continue
        rot_ref = rot @ frac[0]
        trans = []
        for j in range(len(frac)):  # find_translations: candidates from atom 0
            if species[j] != species[0]:
                continue
            t = _wrap01(frac[j] - rot_ref)
            if any(_frac_close(t, u, tol) for u in trans):
                continue
            ok = True
            for i in range(len(frac)):  # translation_valid
                target = rot @ frac[i] + t
                if not any(species[k] == species[i] and _frac_close(target, frac[k], tol) for k in range(len(frac))):
                    ok = False
                    break
            if ok:
                trans.append(t)
        if not trans:
            continue
        k_rot = np.rint(np.linalg.inv(rot).T).astype(np.int64)
        for t in trans:
            if any(np.array_equal(rot, r) and _frac_close(t, u, tol) for r, _, u in ops):  # has_sym_op
                continue
            ops.append((rot, k_rot, t))
    return ops


def _freqs(n):
    i = np.arange(n)
    half = (n - 1) // 2
    return np.where(i <= half, i, i - n)  # fft_grid.zig:434-438


def symmetrize_density(rho, dims, ops, phase_tol=1e-12):
    """rho(G) -> (1/|ops|) sum_op rho(k_rot G) e^{-2 pi i frac(G . t)} (the phase only where frac(G.t)
    is not within phase_tol of an integer), G the signed Miller indices of the grid, then back to
    real space.  rho: N values, x fastest; dims = (nx, ny, nz)."""
    nx, ny, nz = dims
    if len(ops) <= 1:
        return np.asarray(rho, dtype=np.float64).copy()
    rg = op.to_g(rho, dims).reshape(nz, ny, nx)
    h = _freqs(nx)[None, None, :]
    k = _freqs(ny)[None, :, None]
    l = _freqs(nz)[:, None, None]
    out = np.zeros_like(rg)
    for _, kr, t in ops:
        hh = kr[0, 0] * h + kr[0, 1] * k + kr[0, 2] * l
        kk = kr[1, 0] * h + kr[1, 1] * k + kr[1, 2] * l
        ll = kr[2, 0] * h + kr[2, 1] * k + kr[2, 2] * l
        term = rg[np.mod(ll, nz), np.mod(kk, ny), np.mod(hh, nx)]
        dot = h * t[0] + k * t[1] + l * t[2]
        fr = dot - np.floor(dot)
        ph = np.where((fr > phase_tol) & (fr < 1.0 - phase_tol), np.exp(-2j * math.pi * fr), 1.0)
        out += term * ph
    out /= len(ops)
    return op.to_r(out.ravel(), dims)
