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


class OracleBackend:
    """The SCF driver's backend interface (dft-zig_b200/scf.py) implemented with the oracle:
    oracle H|psi> (apply.zig), oracle Davidson (serial.zig) and oracle density (kpoint/density.zig)."""

    def __init__(self):
        self.ctxs = []

    def setup(self, kinputs):
        from oracle.apply import ApplyContext, Atom
        from oracle.pseudo import NonlocalSpecies
        from oracle.pw import Basis, Grid

        for inp in kinputs:
            b = inp.basis
            basis = Basis(hkl=b.hkl, cart=b.gcart, kpg=b.kpg, kinetic=b.kinetic)
            grid = Grid(inp.dims[0], inp.dims[1], inp.dims[2], inp.volume)
            nl = []
            for s, (l_list, dij, phi) in enumerate(inp.species_phi):
                offs, cnts, tot = [], [], 0
                for l in l_list:
                    offs.append(tot)
                    cnts.append(2 * l + 1)
                    tot += 2 * l + 1
                nl.append(NonlocalSpecies(s, list(l_list), offs, cnts, tot, np.asarray(dij), np.asarray(phi)))
            atoms = [Atom(int(sp), np.asarray(pos)) for sp, pos in zip(inp.atom_species, inp.positions)]
            self.ctxs.append(ApplyContext(grid, basis, np.zeros(grid.count), nl, atoms, inp.volume))

    def set_vloc(self, local_r):
        for c in self.ctxs:
            c.local_r = np.asarray(local_r, dtype=np.float64)

    def eig(self, k, diag, nbands, opts, init):
        from oracle import lobpcg

        c = self.ctxs[k]
        r = lobpcg.solve(lobpcg.Operator(c.n, c.apply_batch), diag, nbands, lobpcg.Options(**opts, init_vectors=init))
        return r.values, r.vectors

    def density(self, k, vectors, weights, rho):
        from oracle import density as odens

        c = self.ctxs[k]
        rho += odens.accumulate_density(c.grid, c.map, np.asarray(vectors), np.asarray(weights), c.inv_volume)

    def close(self):
        self.ctxs = []
