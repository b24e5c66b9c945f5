"""Shared builders for the parity tests: seeded k-point problems from the oracle's synthetic cells."""
from __future__ import annotations

import functools

import numpy as np

from oracle import cases


@functools.lru_cache(maxsize=None)
def cell(name: str, seed: int = 1):
    return cases.make_cell(name, seed)


@functools.lru_cache(maxsize=None)
def kproblem(name: str, ecut: float, k_frac=(0.0, 0.0, 0.0), seed: int = 1):
    return cases.make_kproblem(cell(name, seed), ecut, k_frac)


def random_block(n: int, ncols: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(ncols, n)) + 1j * rng.normal(size=(ncols, n))).astype(np.complex128)


def rel_err(a, b) -> float:
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def make_context(dz, kp, precision=0):
    ctx = kp.ctx
    kc = dz.KpointContext.from_basis((kp.grid.nx, kp.grid.ny, kp.grid.nz), kp.grid.volume, ctx.basis, precision)
    kc.set_vloc(ctx.local_r)
    if ctx.nl:
        species = [dz.SpeciesProjectors(ns.l_list, ns.dij, ns.phi) for ns in ctx.nl]
        kc.set_projectors(species, [a.species_index for a in ctx.atoms], np.array([a.position for a in ctx.atoms]))
    return kc
