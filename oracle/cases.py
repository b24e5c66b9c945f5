"""Seeded synthetic cells and one-k-point H|psi> problems (oracle; test infrastructure only).

Cells follow the workloads the hot path is measured on:
  si2    Si diamond FCC primitive cell, a = 5.431 A, atoms at 0 and (1/4,1/4,1/4)a
         (benchmarks/silicon/silicon.xyz and dft_zig_lobpcg_test_serial.toml [cell])
  si8    8-atom conventional cubic Si cell (examples/silicon.xyz)
  si64   2x2x2 supercell of si8 with seeded N(0, 0.02 A) displacements
  si216  3x3x3 supercell of si8 with seeded N(0, 0.05 A) displacements
  al4    FCC Al conventional cell a = 4.05 A with a seeded symmetric strain in [-1%, 1%]
  sige8  8-atom zincblende-type Si(1-x)Ge(x) cell, a = 5.43 + 0.23 x A, +-2% strain

The local potential V(r) = Re N IFFT(sum_s S_s(G) v_s(|G|)) uses the short-range local
form factor of each species' radial mesh (local_vq_short_range, form_factor.zig:223-262)
on |G|^2 < 4 ecut, with V(G=0) = 0, built like build_local_potential_real
(src/features/scf/potential.zig:320-334).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import fft as offt
from .apply import ApplyContext, Atom
from .pseudo import Species, build_nonlocal_species, ionic_potential_radial, radial_tables, synthetic_species
from .pw import ANGSTROM_TO_BOHR, Grid, auto_grid, build_fft_index_map, cell_volume, generate_basis, index_to_freq, reciprocal

SI8_FRAC = np.array(
    [
        [0.0, 0.0, 0.0],
        [0.0, 0.5, 0.5],
        [0.5, 0.0, 0.5],
        [0.5, 0.5, 0.0],
        [0.25, 0.25, 0.25],
        [0.25, 0.75, 0.75],
        [0.75, 0.25, 0.75],
        [0.75, 0.75, 0.25],
    ]
)
FCC4_FRAC = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])


@dataclass
class Cell:
    name: str
    cell: np.ndarray  # rows a_i, bohr
    species: list  # [Species]
    atoms: list  # [Atom] (Cartesian bohr)

    @property
    def recip(self):
        return reciprocal(self.cell)

    @property
    def volume(self):
        return cell_volume(self.cell)

    @property
    def nelec(self):
        return float(sum(self.species[a.species_index].z_val for a in self.atoms))


def _supercell(a_ang: float, frac: np.ndarray, reps: int, sigma_ang: float, seed: int, names, occupancy=None):
    a = a_ang * ANGSTROM_TO_BOHR
    cell = np.eye(3) * a * reps
    pos = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                for f in frac:
                    pos.append((np.array([i, j, k]) + f) * a)
    pos = np.array(pos)
    rng = np.random.default_rng(seed)
    if sigma_ang > 0.0:
        pos = pos + rng.normal(0.0, sigma_ang * ANGSTROM_TO_BOHR, size=pos.shape)
    return cell, pos


def make_cell(name: str, seed: int = 0) -> Cell:
    si = synthetic_species("Si")
    if name == "si2":
        h = 5.431 * ANGSTROM_TO_BOHR / 2.0
        cell = np.array([[0.0, h, h], [h, 0.0, h], [h, h, 0.0]])
        atoms = [Atom(0, np.zeros(3)), Atom(0, np.array([h / 2.0, h / 2.0, h / 2.0]))]
        return Cell(name, cell, [si], atoms)
    if name in ("si8", "si64", "si216"):
        reps, sigma = {"si8": (1, 0.0), "si64": (2, 0.02), "si216": (3, 0.05)}[name]
        cell, pos = _supercell(5.431, SI8_FRAC, reps, sigma, seed, None)
        return Cell(name, cell, [si], [Atom(0, p) for p in pos])
    if name == "al4":
        al = synthetic_species("Al")
        rng = np.random.default_rng(seed)
        e = rng.uniform(-0.01, 0.01, size=(3, 3))
        e = 0.5 * (e + e.T)
        a = 4.05 * ANGSTROM_TO_BOHR
        cell = (np.eye(3) * a) @ (np.eye(3) + e)
        pos = FCC4_FRAC @ cell
        return Cell(name, cell, [al], [Atom(0, p) for p in pos])
    if name == "sige8":
        ge = synthetic_species("Ge")
        rng = np.random.default_rng(seed)
        x = rng.uniform(0.0, 1.0)
        a = (5.43 + 0.23 * x) * ANGSTROM_TO_BOHR
        e = rng.uniform(-0.02, 0.02, size=(3, 3))
        e = 0.5 * (e + e.T)
        cell = (np.eye(3) * a) @ (np.eye(3) + e)
        occ = rng.uniform(0.0, 1.0, size=8) < x
        pos = SI8_FRAC @ cell
        atoms = [Atom(1 if occ[i] else 0, pos[i]) for i in range(8)]
        return Cell(name, cell, [si, ge], atoms)
    raise KeyError(name)


def local_potential_r(c: Cell, grid: Grid, ecut_ry: float) -> np.ndarray:
    """V(r) on the FFT-order grid: the ionic potential of the species' radial meshes with the
    reference's short-range form factor (pseudo.ionic_potential_radial), |G|^2 < 4 ecut, V(0) = 0."""
    meshes = [(sp.r, sp.rab, sp.vloc_r, sp.z_val) for sp in c.species]
    vg, _ = ionic_potential_radial(meshes, [a.species_index for a in c.atoms], [a.position for a in c.atoms],
                                   (grid.nx, grid.ny, grid.nz), c.recip, c.volume, 4.0 * ecut_ry)
    vr = offt.fft3d_inverse(vg * grid.count, grid.nx, grid.ny, grid.nz)
    return vr.real.copy()


@dataclass
class KProblem:
    cell: Cell
    ecut_ry: float
    k_frac: np.ndarray
    grid: Grid
    ctx: ApplyContext
    tables: list


def make_kproblem(c: Cell, ecut_ry: float, k_frac=(0.0, 0.0, 0.0), grid_dims=None, local_r=None, tables=None) -> KProblem:
    recip = c.recip
    dims = grid_dims or auto_grid(ecut_ry, recip)
    grid = Grid(dims[0], dims[1], dims[2], c.volume)
    k_cart = np.asarray(k_frac, dtype=np.float64) @ recip
    basis = generate_basis(recip, ecut_ry, k_cart)
    if tables is None:
        tables = [radial_tables(sp, ecut_ry) for sp in c.species]
    nl = [build_nonlocal_species(s, sp, basis.kpg, tables[s]) for s, sp in enumerate(c.species)]
    if local_r is None:
        local_r = local_potential_r(c, grid, ecut_ry)
    ctx = ApplyContext(grid, basis, local_r, nl, c.atoms, c.volume)
    return KProblem(c, ecut_ry, np.asarray(k_frac, dtype=np.float64), grid, ctx, tables)


def monkhorst_pack(mesh):
    """Unshifted Gamma-centred MP grid in fractional coordinates, with k and -k folded together
    (time reversal).  Weights sum to 1."""
    n1, n2, n3 = mesh
    pts = {}
    order = []
    for i in range(n1):
        for j in range(n2):
            for k in range(n3):
                key = (i, j, k)
                neg = ((-i) % n1, (-j) % n2, (-k) % n3)
                if neg in pts:
                    pts[neg][1] += 1
                else:
                    f = np.array([i / n1, j / n2, k / n3])
                    f = np.where(f > 0.5, f - 1.0, f)
                    pts[key] = [f, 1]
                    order.append(key)
    tot = n1 * n2 * n3
    return [(pts[key][0], pts[key][1] / tot) for key in order]
