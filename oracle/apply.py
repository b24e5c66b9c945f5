"""H|psi> = (T + V_loc + V_nl)|psi> for one k-point (oracle; test infrastructure only).

Restates src/features/scf/apply.zig:
  577-641   apply_hamiltonian_with_workspace (single column: kinetic, local, nonlocal)
  811-880   apply_local_potential_safe (fused path: scatter_fft(xN) -> inverse FFT(/N) -> x V(r)
            -> forward FFT -> gather_fft(x1/N))
  883-896   compute_atom_phase: phase_g = exp(i G_g . tau)   (G, not k+G)
  899-1037  scalar projector path (project, D_ij, back-project with conj(phase)/Omega)
  1118-1336 batched projector path (re/im dgemm formulation)
  1584-1618 apply_hamiltonian_batched

Arrays of columns are stored as numpy ``(ncols, n)`` which is the reference's
column-major ``[n x ncols]`` complex128 layout (lobpcg/common.zig:16-24).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import fft as offt
from .pw import Basis, Grid, PwGridMap, build_fft_index_map


@dataclass
class Atom:
    species_index: int
    position: np.ndarray  # Cartesian bohr


class ApplyContext:
    """The parts of apply.zig ApplyContext (45-169) the hot path reads."""

    def __init__(self, grid: Grid, basis: Basis, local_r: np.ndarray, nonlocal_species, atoms, volume: float):
        self.grid = grid
        self.basis = basis
        self.local_r = np.asarray(local_r, dtype=np.float64)
        self.nl = list(nonlocal_species) if nonlocal_species else []
        self.atoms = list(atoms)
        self.inv_volume = 1.0 / volume
        self.map = PwGridMap(basis, grid)
        self.map.build_fft_indices(build_fft_index_map(grid))

    @property
    def n(self):
        return self.basis.n

    # -- local potential ---------------------------------------------------
    def apply_local(self, x: np.ndarray) -> np.ndarray:
        g = self.grid
        total = float(g.count)
        work = np.zeros(g.count, dtype=np.complex128)
        self.map.scatter_fft(x, work, total)
        work = offt.fft3d_inverse(work, g.nx, g.ny, g.nz)
        work = work * self.local_r
        work = offt.fft3d_forward(work, g.nx, g.ny, g.nz)
        return self.map.gather_fft(work, 1.0 / total)

    # -- nonlocal (scalar) -------------------------------------------------
    def apply_nonlocal(self, x: np.ndarray) -> np.ndarray:
        """apply.zig:999-1037 with the sequential loops written as matrix products."""
        out = np.zeros(self.n, dtype=np.complex128)
        for entry in self.nl:
            if entry.m_total == 0:
                continue
            from .pseudo import expand_dij_m

            dm = expand_dij_m(entry)
            for atom in self.atoms:
                if atom.species_index != entry.species_index:
                    continue
                phase = np.exp(1j * (self.basis.cart @ atom.position))
                coeff = entry.phi @ (x * phase)
                coeff2 = dm @ coeff
                out += np.conj(phase) * (entry.phi.T @ coeff2) * self.inv_volume
        return out

    # -- nonlocal (batched, dgemm formulation) -----------------------------
    def apply_nonlocal_batched(self, xb: np.ndarray) -> np.ndarray:
        """apply.zig:1118-1336,1454-1482: per atom, xphase split into re/im row-major [n_pw x ncols],
        coeffs = phi . xphase (2 dgemm), coeffs2 = D coeffs, r = phi^T coeffs2 (2 dgemm),
        out += conj(phase) r / Omega."""
        ncols = xb.shape[0]
        out = np.zeros((ncols, self.n), dtype=np.complex128)
        from .pseudo import expand_dij_m

        for entry in self.nl:
            if entry.m_total == 0:
                continue
            dm = expand_dij_m(entry)
            for atom in self.atoms:
                if atom.species_index != entry.species_index:
                    continue
                phase = np.cos(self.basis.cart @ atom.position) + 1j * np.sin(self.basis.cart @ atom.position)
                xphase = (xb * phase[None, :]).T  # [n_pw, ncols]
                c_re = entry.phi @ xphase.real
                c_im = entry.phi @ xphase.imag
                c2_re = dm @ c_re
                c2_im = dm @ c_im
                r_re = entry.phi.T @ c2_re
                r_im = entry.phi.T @ c2_im
                ph = np.conj(phase)[:, None]
                add = (ph.real * r_re - ph.imag * r_im) * self.inv_volume + 1j * (
                    (ph.real * r_im + ph.imag * r_re) * self.inv_volume
                )
                out += add.T
        return out

    # -- full H ------------------------------------------------------------
    def apply(self, x: np.ndarray) -> np.ndarray:
        """apply.zig:577-641."""
        y = x * self.basis.kinetic
        y = y + self.apply_local(x)
        if self.nl:
            y = y + self.apply_nonlocal(x)
        return y

    def apply_batch(self, xb: np.ndarray) -> np.ndarray:
        """apply.zig:1584-1618: per-column kinetic + local, then batched nonlocal."""
        xb = np.asarray(xb, dtype=np.complex128).reshape(-1, self.n)
        yb = np.empty_like(xb)
        for c in range(xb.shape[0]):
            yb[c] = xb[c] * self.basis.kinetic + self.apply_local(xb[c])
        if self.nl:
            yb = yb + self.apply_nonlocal_batched(xb)
        return yb

    def nonlocal_energy(self, psi: np.ndarray) -> float:
        """kpoint/density.zig:145-165: Re <psi|V_nl|psi> via the scalar projector path."""
        return float(np.vdot(psi, self.apply_nonlocal(psi)).real)

    def dense_hamiltonian(self) -> np.ndarray:
        """Dense H built column by column from apply() (the role of apply.zig:660-729's
        check against hamiltonian.build_hamiltonian, used only on tiny bases)."""
        n = self.n
        h = np.zeros((n, n), dtype=np.complex128)
        e = np.zeros(n, dtype=np.complex128)
        for j in range(n):
            e[:] = 0
            e[j] = 1.0
            h[:, j] = self.apply(e)
        return h
