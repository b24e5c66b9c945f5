"""Host-side inputs of the hot path: cells, plane-wave basis, FFT box, projector tables, V_loc(r).

In the reference these come from the SCF driver that calls the path (outside its scope):
  plane_wave/basis.zig:26-74            G-sphere per k (h outer, l inner; |k+G|^2 <= ecut)
  scf/pw_grid.zig:54-72, fft/sizing.zig auto FFT box (next 2,3,5-smooth >= 2 ceil(2 sqrt(ecut)/|b|) + 1)
  pseudopotential/nonlocal.zig:8-338    radial projector tables (ctrap weights, j_l, 2048-point table)
  scf/nonlocal_context.zig:387-549      phi = 4 pi R(|k+G|) Y_lm(k+G)
  scf/potential.zig:320-334             V(r) = Re N IFFT(V(G))
This module builds them with vectorised numpy for the benchmark and SCF workloads.  The synthetic
species use the Goedecker-Teter-Hutter functional form with builder-chosen parameters (the
reference ships no pseudopotential files); they are not a published pseudopotential.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

BOHR_PER_ANGSTROM = 1.0 / 0.529177210903

# Builder-chosen GTH-form parameters (energies in Hartree): Z, r_loc, C1, C2 and per channel
# (l, r_l, h matrix).
SPECIES_PARAMS = {
    "Si": dict(z=4.0, rloc=0.44, c1=-7.34, c2=0.0, chans=[(0, 0.423, [[5.9, 0.0], [0.0, 2.0]]), (1, 0.484, [[2.73]])]),
    "Al": dict(z=3.0, rloc=0.45, c1=-8.5, c2=0.0, chans=[(0, 0.46, [[5.1, 0.0], [0.0, 1.2]]), (1, 0.54, [[2.2]])]),
    "Ge": dict(z=4.0, rloc=0.54, c1=0.0, c2=0.0, chans=[(0, 0.42, [[7.5, 0.0], [0.0, 2.4]]), (1, 0.56, [[2.5]])]),
}

DIAMOND8 = np.array(
    [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0], [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25]]
)
FCC4 = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]])


@dataclass
class SpeciesData:
    """UPF-shaped arrays of one species."""

    name: str
    z_val: float
    r: np.ndarray
    rab: np.ndarray
    betas: list  # (l, r*beta(r))
    dij: np.ndarray  # Ry
    params: dict = field(default_factory=dict)
    vloc: np.ndarray = None  # local potential on the mesh (Ry), the UPF's PP_LOCAL

    @property
    def mesh(self):
        """(r, rab, vloc, z_valence): the inputs of the radial local form factor."""
        return (self.r, self.rab, self.vloc, self.z_val)


def log_mesh(zmesh=14.0, xmin=-7.0, dx=0.0125, rmax=10.0):
    n = int((math.log(zmesh * rmax) - xmin) / dx) + 1
    r = np.exp(xmin + np.arange(n) * dx) / zmesh
    return r, r * dx


def species(name: str) -> SpeciesData:
    p = SPECIES_PARAMS[name]
    r, rab = log_mesh()
    betas, blocks = [], []
    for l, rl, h in p["chans"]:
        h = np.asarray(h, float)
        for i in range(1, h.shape[0] + 1):
            e = l + (4.0 * i - 1.0) / 2.0
            proj = math.sqrt(2.0) * r ** (l + 2 * (i - 1)) * np.exp(-(r * r) / (2 * rl * rl)) / (rl**e * math.sqrt(math.gamma(e)))
            betas.append((l, r * proj))
        blocks.append(h)
    nb = len(betas)
    dij = np.zeros((nb, nb))
    o = 0
    for h in blocks:
        k = h.shape[0]
        dij[o : o + k, o : o + k] = 2.0 * h
        o += k
    # the GTH local potential tabulated on the mesh, Hartree -> Ry
    from scipy.special import erf

    rl = p["rloc"]
    vloc = 2.0 * (-p["z"] / r * erf(r / (math.sqrt(2.0) * rl)) + np.exp(-0.5 * (r / rl) ** 2) * (p["c1"] + p["c2"] * (r / rl) ** 2))
    return SpeciesData(name, p["z"], r, rab, betas, dij, p, vloc)


@dataclass
class Crystal:
    cell: np.ndarray  # bohr, rows
    species: list  # [SpeciesData]
    atom_species: np.ndarray  # int
    positions: np.ndarray  # bohr, Cartesian [natom,3]

    @property
    def recip(self):
        a1, a2, a3 = self.cell
        v = float(np.dot(a1, np.cross(a2, a3)))
        return 2.0 * math.pi / v * np.array([np.cross(a2, a3), np.cross(a3, a1), np.cross(a1, a2)])

    @property
    def volume(self):
        return abs(float(np.linalg.det(self.cell)))

    @property
    def nelec(self):
        return float(sum(self.species[s].z_val for s in self.atom_species))


def crystal(name: str, seed: int = 1) -> Crystal:
    """The benchmark cells (same constructions and seeds as the parity tests)."""
    si = species("Si")
    if name == "si2":
        h = 5.431 * BOHR_PER_ANGSTROM / 2.0
        cell = np.array([[0.0, h, h], [h, 0.0, h], [h, h, 0.0]])
        return Crystal(cell, [si], np.zeros(2, int), np.array([[0.0, 0.0, 0.0], [h / 2, h / 2, h / 2]]))
    if name in ("si8", "si64", "si216"):
        reps, sigma = {"si8": (1, 0.0), "si64": (2, 0.02), "si216": (3, 0.05)}[name]
        a = 5.431 * BOHR_PER_ANGSTROM
        shifts = np.array([[i, j, k] for i in range(reps) for j in range(reps) for k in range(reps)], float)
        pos = ((shifts[:, None, :] + DIAMOND8[None, :, :]).reshape(-1, 3)) * a
        rng = np.random.default_rng(seed)
        if sigma > 0:
            pos = pos + rng.normal(0.0, sigma * BOHR_PER_ANGSTROM, size=pos.shape)
        return Crystal(np.eye(3) * a * reps, [si], np.zeros(len(pos), int), pos)
    if name == "si8d":
        # training / evaluation cells of the learned preconditioner: the 8-atom cubic cell with a
        # seeded symmetric strain in [-1%, 1%] and N(0, 0.05 A) displacements
        rng = np.random.default_rng(seed)
        e = rng.uniform(-0.01, 0.01, size=(3, 3))
        e = 0.5 * (e + e.T)
        cell = (np.eye(3) * 5.431 * BOHR_PER_ANGSTROM) @ (np.eye(3) + e)
        pos = DIAMOND8 @ cell + rng.normal(0.0, 0.05 * BOHR_PER_ANGSTROM, size=(8, 3))
        return Crystal(cell, [si], np.zeros(8, int), pos)
    if name in ("sitrain", "sival"):
        # the learned preconditioner's training and held-out cells: 8 to 64 Si atoms (supercells
        # of the 8-atom cubic cell, shape drawn from the seed), a seeded symmetric strain in
        # [-1%, 1%] and N(0, 0.05 A) displacements; "sival": its 144-atom (3 x 3 x 2) validation cells
        rng = np.random.default_rng(seed)
        shapes = [(1, 1, 1), (2, 1, 1), (3, 1, 1), (2, 2, 1), (3, 2, 1), (2, 2, 2)]
        pick = int(rng.integers(0, len(shapes)))
        reps = np.array(shapes[pick] if name == "sitrain" else (3, 3, 2))
        e = rng.uniform(-0.01, 0.01, size=(3, 3))
        e = 0.5 * (e + e.T)
        a = 5.431 * BOHR_PER_ANGSTROM
        cell = (np.diag(reps.astype(float)) * a) @ (np.eye(3) + e)
        shifts = np.array([[i, j, k] for i in range(reps[0]) for j in range(reps[1]) for k in range(reps[2])], float)
        frac = ((shifts[:, None, :] + DIAMOND8[None, :, :]).reshape(-1, 3)) / reps
        pos = frac @ cell + rng.normal(0.0, 0.05 * BOHR_PER_ANGSTROM, size=(len(frac), 3))
        return Crystal(cell, [si], np.zeros(len(pos), int), pos)
    if name == "al4":
        rng = np.random.default_rng(seed)
        e = rng.uniform(-0.01, 0.01, size=(3, 3))
        e = 0.5 * (e + e.T)
        cell = (np.eye(3) * 4.05 * BOHR_PER_ANGSTROM) @ (np.eye(3) + e)
        return Crystal(cell, [species("Al")], np.zeros(4, int), FCC4 @ cell)
    if name == "sige8":
        rng = np.random.default_rng(seed)
        x = rng.uniform(0.0, 1.0)
        a = (5.43 + 0.23 * x) * BOHR_PER_ANGSTROM
        e = rng.uniform(-0.02, 0.02, size=(3, 3))
        e = 0.5 * (e + e.T)
        cell = (np.eye(3) * a) @ (np.eye(3) + e)
        occ = rng.uniform(0.0, 1.0, size=8) < x
        return Crystal(cell, [si, species("Ge")], occ.astype(int), DIAMOND8 @ cell)
    raise KeyError(name)


# Width (bohr) of the Gaussian atomic valence density of the synthetic species (the UPF PP_RHOATOM
# they lack): rho_atom(r) = Z / (pi^{3/2} a^3) exp(-r^2 / a^2), form factor Z exp(-G^2 a^2 / 4).
ATOM_DENSITY_WIDTH = {"Si": 1.55, "Ge": 1.65, "Al": 1.75}


def atomic_density_channels(c: "Crystal", dims) -> np.ndarray:
    """Superposition of atomic valence densities on the FFT grid (x fastest), one channel per
    species group: [0] all species except Ge, [1] Ge.  build_atomic_density (scf/core_density.zig:
    128-183): rho(G) = (1/Omega) sum_atoms f(|G|) exp(-i G . R), inverse FFT to real space."""
    nx, ny, nz = dims
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    hkl = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1)
    G = hkl @ c.recip
    g2 = (G * G).sum(axis=1)
    out = np.zeros((2, nx * ny * nz))
    for ch in range(2):
        rho_g = np.zeros(nx * ny * nz, dtype=np.complex128)
        for a, s in enumerate(c.atom_species):
            sp = c.species[s]
            if (sp.name == "Ge") != (ch == 1):
                continue
            w = ATOM_DENSITY_WIDTH.get(sp.name, 1.6)
            rho_g += sp.z_val * np.exp(-g2 * w * w / 4.0) * np.exp(-1j * (G @ c.positions[a]))
        rho_g /= c.volume
        out[ch] = np.fft.ifftn(rho_g.reshape(nz, ny, nx)).ravel().real * (nx * ny * nz)
    return out


def _smooth235(n):
    m = n
    for p in (2, 3, 5):
        while m % p == 0:
            m //= p
    return m == 1


def fft_box(ecut: float, recip: np.ndarray):
    out = []
    for i in range(3):
        n = max(int(math.ceil(2.0 * math.sqrt(ecut) / float(np.linalg.norm(recip[i])))) * 2 + 1, 3)
        while not _smooth235(n):
            n += 1
        out.append(n)
    return tuple(out)


@dataclass
class PwBasis:
    hkl: np.ndarray
    gcart: np.ndarray
    kpg: np.ndarray
    kinetic: np.ndarray

    @property
    def n(self):
        return int(self.kinetic.size)


def basis(recip: np.ndarray, ecut: float, k_frac) -> PwBasis:
    k = np.asarray(k_frac, float) @ recip
    nmax = int(math.ceil(math.sqrt(ecut) / min(np.linalg.norm(recip, axis=1)))) + 1
    r = np.arange(-nmax, nmax + 1)
    hkl = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    g = (recip[0] * hkl[:, :1] + recip[1] * hkl[:, 1:2]) + recip[2] * hkl[:, 2:3]
    kpg = k + g
    kin = kpg[:, 0] ** 2 + kpg[:, 1] ** 2 + kpg[:, 2] ** 2
    sel = kin <= ecut
    return PwBasis(hkl[sel].astype(np.int32), g[sel], kpg[sel], kin[sel])


def _sph_jl(l: int, x: np.ndarray) -> np.ndarray:
    small = np.abs(x) < 1e-6
    xs = np.where(small, 1.0, x)  # keeps the closed form finite where the series is used
    if l == 0:
        return np.where(small, 1.0 - x**2 / 6.0 + x**4 / 120.0, np.sin(xs) / xs)
    if l == 1:
        return np.where(small, x / 3.0 - x**3 / 30.0, np.sin(xs) / (xs * xs) - np.cos(xs) / xs)
    raise NotImplementedError("synthetic species carry l <= 1 projectors")


def radial_table(sp: SpeciesData, b: int, ecut: float, npts: int = 2048) -> tuple:
    """Uniform table of R_b(q) = sum_i r_i (r beta)_i j_l(q r_i) rab_i w_i over [0, 1.5 sqrt(2 ecut)]."""
    l, beta = sp.betas[b]
    gmax = 1.5 * math.sqrt(2.0 * ecut)
    dq = gmax / (npts - 1)
    q = dq * np.arange(npts)
    n = sp.r.size
    w = np.ones(n)
    if n >= 10:
        cw = np.array([23.75, 95.10, 55.20, 79.30, 70.65]) / 72.0
        w[:5] = cw
        w[-5:] = cw[::-1]
    f = sp.r * beta * sp.rab * w
    vals = np.cumsum(_sph_jl(l, np.outer(q, sp.r)) * f[None, :], axis=1)[:, -1]
    return vals, gmax, dq


def _interp(table, g):
    vals, gmax, dq = table
    x = g / dq
    i = np.floor(x).astype(np.int64)
    t = x - i
    out = np.zeros_like(g)
    inside = (g > 0) & (g < gmax)
    last = inside & (i + 1 >= vals.size)
    mid = inside & ~last
    out[mid] = vals[i[mid]] * (1 - t[mid]) + vals[i[mid] + 1] * t[mid]
    out[last] = vals[-1]
    out[g <= 0] = vals[0]
    return out


def _ylm(l, m, v):
    r = np.sqrt((v * v).sum(axis=1))
    zero = r < math.sqrt(1e-30)
    u = v / np.where(zero, 1.0, r)[:, None]
    if l == 0:
        return np.full(len(v), 1.0 / math.sqrt(4 * math.pi))
    c = math.sqrt(3.0 / (4 * math.pi))
    y = c * u[:, {-1: 1, 0: 2, 1: 0}[m]]
    return np.where(zero, 0.0, y)


def projectors(sp: SpeciesData, kpg: np.ndarray, tables) -> np.ndarray:
    """phi[m_total, n_pw] for one species."""
    g = np.sqrt((kpg * kpg).sum(axis=1))
    rows = []
    for b, (l, _) in enumerate(sp.betas):
        rad = _interp(tables[b], g)
        for mi in range(2 * l + 1):
            rows.append(4.0 * math.pi * rad * _ylm(l, mi - l, kpg))
    return np.array(rows)


def _interp_deriv(table, g):
    """dR/dq from the table as RadialTable.eval_deriv (pseudopotential/nonlocal.zig:294-299): a central
    difference of the interpolant with the table step, one-sided below the first step."""
    _, _, dq = table
    fwd = (_interp(table, np.full_like(g, dq)) - _interp(table, np.zeros_like(g))) / dq
    cen = (_interp(table, g + dq) - _interp(table, g - dq)) / (2.0 * dq)
    return np.where(g < dq, fwd, cen)


def _dylm(l, m, v):
    """Gradient of Y_lm(v / |v|) with respect to v (stress/stress.zig:79-107): zero for l = 0 and at
    |v| < 1e-15; for l = 1, c (e_j - n n_j) / |v| with Y_1m = c n_j."""
    out = np.zeros_like(v)
    if l == 0:
        return out
    r = np.sqrt((v * v).sum(axis=1))
    ok = r >= 1e-15
    inv = np.where(ok, 1.0 / np.where(ok, r, 1.0), 0.0)
    u = v * inv[:, None]
    j = {-1: 1, 0: 2, 1: 0}[m]
    c = math.sqrt(3.0 / (4 * math.pi))
    out = -c * u * u[:, j:j + 1]
    out[:, j] += c
    return out * inv[:, None]


def projector_derivatives(sp: SpeciesData, kpg: np.ndarray, tables) -> np.ndarray:
    """dphi[m_total, 3, n_pw] = d phi_bm / d q_a = 4 pi (R_b'(|q|) q_a / |q| Y_lm + R_b dY_lm/dq_a) for
    one species, zero where |q| < 1e-12: the derivative projectors of the nonlocal stress
    (project_p_and_dp, stress/nonlocal_stress.zig:108-165)."""
    g = np.sqrt((kpg * kpg).sum(axis=1))
    live = g >= 1e-12
    nhat = kpg * np.where(live, 1.0 / np.where(live, g, 1.0), 0.0)[:, None]
    rows = []
    for b, (l, _) in enumerate(sp.betas):
        rad, drad = _interp(tables[b], g), _interp_deriv(tables[b], g)
        for mi in range(2 * l + 1):
            y = _ylm(l, mi - l, kpg)
            d = 4.0 * math.pi * (drad[:, None] * nhat * y[:, None] + rad[:, None] * _dylm(l, mi - l, kpg))
            rows.append((d * live[:, None]).T)
    return np.array(rows)


def local_form_factor(sp: SpeciesData, q: np.ndarray) -> np.ndarray:
    """The reference's local form factor in its default short_range mode (local_vq_short_range,
    pseudopotential/form_factor.zig:223-262), Ry: 4 pi sum_j r_j^2 [V_loc(r_j) + 2 Z / r_j]
    sinc(q r_j) rab_j w_j - 8 pi Z / q^2, the Coulomb term left out at q < 1e-10 (so V(0) is epsatm)."""
    r, rab, vloc, z = sp.mesh
    n = r.size
    w = np.ones(n)
    if n >= 10:
        cw = np.array([23.75, 95.10, 55.20, 79.30, 70.65]) / 72.0
        w[:5] = cw
        w[n - 5:] = cw[::-1]
    vc = np.where(r < 1e-10, 0.0, 2.0 * z / np.where(r < 1e-10, 1.0, r))
    terms = r * r * (vloc + vc) * rab * w
    q = np.atleast_1d(np.asarray(q, dtype=np.float64))
    out = np.empty(q.size)
    for i0 in range(0, q.size, 4096):  # bounded temporaries
        x = np.outer(q[i0:i0 + 4096], r)
        small = np.abs(x) < 1e-12
        out[i0:i0 + 4096] = 4.0 * math.pi * (np.where(small, 1.0, np.sin(x) / np.where(small, 1.0, x)) @ terms)
    big = q >= 1e-10
    out[big] -= 8.0 * math.pi * z / (q[big] * q[big])
    return out


def epsatm(sp: SpeciesData) -> float:
    """compute_epsatm (form_factor.zig:264-268): the q = 0 value of the short-range form factor."""
    return float(local_form_factor(sp, np.zeros(1))[0])


def local_potential(c: Crystal, dims, ecut: float) -> np.ndarray:
    """V(r) (Ry) on the x-fastest box: V(G) = (1/Omega) sum_atoms V_s(|G|) e^{-iG tau} from each
    species' radial mesh (local_form_factor), zero at |G| < 1e-10 and for |G|^2 >= 4 ecut
    (build_ionic_potential_grid, scf/potential.zig:279-318, ecutrho = 4 ecut)."""
    nx, ny, nz = dims
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    gv = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ c.recip
    g2 = (gv * gv).sum(axis=1)
    q = np.sqrt(g2)
    keep = (q >= 1e-10) & (g2 < 4.0 * ecut)
    uq, inv = np.unique(q[keep], return_inverse=True)
    vg = np.zeros(g2.size, complex)
    for s, sp in enumerate(c.species):
        ff = local_form_factor(sp, uq)[inv]
        sf = np.zeros(keep.sum(), complex)
        for a in np.where(c.atom_species == s)[0]:
            sf += np.exp(-1j * (gv[keep] @ c.positions[a]))
        vg[keep] += sf * ff / c.volume
    n = nx * ny * nz
    return np.fft.ifftn(vg.reshape(nz, ny, nx) * n).real.ravel().copy()


@dataclass
class KpointInputs:
    dims: tuple
    volume: float
    basis: PwBasis
    local_r: np.ndarray
    species_phi: list  # per species: (l_list, dij, phi)
    atom_species: np.ndarray
    positions: np.ndarray


def kpoint_inputs(c: Crystal, ecut: float, k_frac, dims=None, local_r=None, tables=None) -> KpointInputs:
    dims = dims or fft_box(ecut, c.recip)
    b = basis(c.recip, ecut, k_frac)
    if tables is None:
        tables = [[radial_table(sp, i, ecut) for i in range(len(sp.betas))] for sp in c.species]
    sph = [([l for l, _ in sp.betas], sp.dij, projectors(sp, b.kpg, tables[s])) for s, sp in enumerate(c.species)]
    if local_r is None:
        local_r = local_potential(c, dims, ecut)
    return KpointInputs(dims, c.volume, b, local_r, sph, c.atom_species, c.positions)


def kpoint_inputs_device(dz, c: Crystal, ecut: float, k_frac, dims=None, local_r=None, tables=None) -> KpointInputs:
    """kpoint_inputs with the basis (dftcuda_plane_wave_basis, the reference's order and arithmetic)
    and the projector rows 4 pi R(|k+G|) Y_lm (dftcuda_projector_phi) built on the device; tables:
    per species, per beta, (values, gmax, dq) radial tables."""
    dims = dims or fft_box(ecut, c.recip)
    hkl, g, q, kin = dz.plane_wave_basis(c.recip, ecut, np.asarray(k_frac, float) @ c.recip)
    b = PwBasis(hkl, g, q, kin)
    if tables is None:
        tables = [[radial_table(sp, i, ecut) for i in range(len(sp.betas))] for sp in c.species]
    sph = []
    for s, sp in enumerate(c.species):
        rows = [dz.projector_phi(l, tables[s][i], q) for i, (l, _) in enumerate(sp.betas)]
        sph.append(([l for l, _ in sp.betas], sp.dij, np.concatenate(rows, axis=0) if rows else np.zeros((0, len(kin)))))
    if local_r is None:
        local_r = local_potential(c, dims, ecut)
    return KpointInputs(dims, c.volume, b, local_r, sph, c.atom_species, c.positions)


def monkhorst_pack(mesh):
    """Gamma-centred MP mesh, k and -k folded (time reversal).  [(k_frac, weight)]."""
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
