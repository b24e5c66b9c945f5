"""Kleinman-Bylander projector tables and a synthetic norm-conserving pseudopotential
(oracle; test infrastructure only).

Restates:
  src/features/math/radial_integration.zig:7-13     ctrap_weight()
  src/features/pseudopotential/nonlocal.zig:8-21    radial_projector()
  src/features/pseudopotential/nonlocal.zig:59-138  spherical_bessel() (Miller downward recursion)
  src/features/pseudopotential/nonlocal.zig:152-241 real_spherical_harmonic() l <= 4
  src/features/pseudopotential/nonlocal.zig:250-338 RadialTable / RadialTableSet (2048 points)
  src/features/scf/nonlocal_context.zig:387-549     NonlocalSpecies (l_list, m_offsets, phi)
  src/features/scf/common.zig:124-149               table g_max = 1.5*sqrt(2*ecut)  (the call site)

The reference ships no UPF file (pseudo/README.md:4), so ``synthetic_species``
builds UPF-shaped arrays (r, rab, r*beta(r), D_ij, V_loc(r)) from the analytic
Goedecker-Teter-Hutter functional form with builder-chosen parameters.  They
are synthetic and are not any published pseudopotential.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

CTRAP_W = np.array([23.75, 95.10, 55.20, 79.30, 70.65]) / 72.0


def ctrap_weights(n: int) -> np.ndarray:
    """radial_integration.zig:7-13 (vectorised)."""
    w = np.ones(n)
    if n < 10:
        return w
    w[:5] = CTRAP_W
    w[n - 5 :] = CTRAP_W[::-1]
    return w


def ctrap_weight(i: int, n: int) -> float:
    return float(ctrap_weights(n)[i])


def _bessel_small(l: int, x: float) -> float:
    x2 = x * x
    if l == 0:
        return 1.0 - x2 / 6.0 + x2 * x2 / 120.0
    if l == 1:
        return x / 3.0 - x * x2 / 30.0
    if l == 2:
        return x2 / 15.0 - x2 * x2 / 210.0
    if l == 3:
        return x * x2 / 105.0
    return 0.0


def _bessel_direct(l: int, x: float) -> float:
    if l > x + 50.0:
        return 0.0
    jlm1 = math.sin(x) / x
    jl = math.sin(x) / (x * x) - math.cos(x) / x
    for n in range(1, l):
        jlp1 = (2.0 * n + 1.0) / x * jl - jlm1
        jlm1, jl = jl, jlp1
        if not math.isfinite(jl):
            return 0.0
    return jl


def _bessel_miller(l: int, x: float) -> float:
    nm = l + 1
    nlim = nm + int(15.0 * x) + 1 if x < 1.0 else nm + int(1.36 * x) + 15
    if nlim > 256:
        return _bessel_direct(l, x)
    sb = [0.0] * (nlim + 2)
    xi = 1.0 / x
    sb[nlim + 1] = 0.0
    sb[nlim] = 1.0e-18
    for n in range(nlim, 0, -1):
        sb[n - 1] = (2.0 * n + 1.0) * xi * sb[n] - sb[n + 1]
    scale = (math.sin(x) / x) / sb[0]
    return sb[nm - 1] * scale


def spherical_bessel(l: int, x: float) -> float:
    """nonlocal.zig:59-71."""
    if abs(x) < 1e-6:
        return _bessel_small(l, x)
    if l == 0:
        return math.sin(x) / x
    if l == 1:
        return math.sin(x) / (x * x) - math.cos(x) / x
    return _bessel_miller(l, x)


def spherical_bessel_vec(l: int, x: np.ndarray) -> np.ndarray:
    """Vectorised spherical_bessel for l <= 1 (exact same formulas); Miller per element otherwise."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = np.abs(x) < 1e-6
    xs = x[small]
    x2 = xs * xs
    if l == 0:
        out[small] = 1.0 - x2 / 6.0 + x2 * x2 / 120.0
        xb = x[~small]
        out[~small] = np.sin(xb) / xb
        return out
    if l == 1:
        out[small] = xs / 3.0 - xs * x2 / 30.0
        xb = x[~small]
        out[~small] = np.sin(xb) / (xb * xb) - np.cos(xb) / xb
        return out
    flat = out.ravel()
    for i, v in enumerate(x.ravel()):
        flat[i] = spherical_bessel(l, float(v))
    return flat.reshape(x.shape)


def radial_projector(beta: np.ndarray, r: np.ndarray, rab: np.ndarray, l: int, g: float) -> float:
    """nonlocal.zig:8-21: sum_i r_i * (r*beta)_i * j_l(g r_i) * rab_i * ctrap_weight(i, n)."""
    n = beta.size
    jl = spherical_bessel_vec(l, g * r)
    terms = r * beta * jl * rab * ctrap_weights(n)
    # cumsum accumulates left to right, the same order as the reference loop.
    return float(np.cumsum(terms)[-1]) if n else 0.0


class RadialTable:
    """nonlocal.zig:250-300: uniform table over [0, g_max] with linear interpolation."""

    def __init__(self, beta, r, rab, l, g_max, n_points=2048):
        n = max(n_points, 2)
        self.dg = g_max / float(n - 1)
        self.g_max = g_max
        self.n_points = n
        self.values = np.array([radial_projector(beta, r, rab, l, self.dg * i) for i in range(n)])

    def eval(self, g: np.ndarray) -> np.ndarray:
        g = np.asarray(g, dtype=np.float64)
        out = np.zeros_like(g)
        x = g / self.dg
        i = np.floor(x).astype(np.int64)
        t = x - i
        inside = (g > 0.0) & (g < self.g_max)
        last = inside & (i + 1 >= self.n_points)
        mid = inside & ~last
        ii = i[mid]
        out[mid] = self.values[ii] * (1.0 - t[mid]) + self.values[ii + 1] * t[mid]
        out[last] = self.values[self.n_points - 1]
        out[g <= 0.0] = self.values[0]
        return out

    def eval_deriv(self, g: np.ndarray) -> np.ndarray:
        """nonlocal.zig:294-299: central difference of eval with the table step; one-sided below dg."""
        g = np.asarray(g, dtype=np.float64)
        fwd = (self.eval(np.full_like(g, self.dg)) - self.eval(np.zeros_like(g))) / self.dg
        cen = (self.eval(g + self.dg) - self.eval(g - self.dg)) / (2.0 * self.dg)
        return np.where(g < self.dg, fwd, cen)


def real_ylm(l: int, m: int, x, y, z) -> np.ndarray:
    """nonlocal.zig:152-241 (vectorised over points)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64)
    r2 = x * x + y * y + z * z
    origin = r2 < 1e-30
    inv_r = 1.0 / np.sqrt(np.where(origin, 1.0, r2))
    nx, ny, nz = x * inv_r, y * inv_r, z * inv_r
    pi = math.pi
    if l == 0:
        v = np.full_like(nx, 1.0 / math.sqrt(4.0 * pi) if m == 0 else 0.0)
    elif l == 1:
        c = math.sqrt(3.0 / (4.0 * pi))
        v = {-1: c * ny, 0: c * nz, 1: c * nx}.get(m, 0.0 * nx)
    elif l == 2:
        c0 = math.sqrt(5.0 / (16.0 * pi))
        c1 = math.sqrt(15.0 / (4.0 * pi))
        c2 = math.sqrt(15.0 / (16.0 * pi))
        v = {
            -2: c2 * 2.0 * nx * ny,
            -1: c1 * ny * nz,
            0: c0 * (3.0 * nz * nz - 1.0),
            1: c1 * nx * nz,
            2: c2 * (nx * nx - ny * ny),
        }.get(m, 0.0 * nx)
    elif l == 3:
        v = {
            -3: math.sqrt(35.0 / (32.0 * pi)) * (3.0 * nx * nx - ny * ny) * ny,
            -2: math.sqrt(105.0 / (4.0 * pi)) * nx * ny * nz,
            -1: math.sqrt(21.0 / (32.0 * pi)) * ny * (5.0 * nz * nz - 1.0),
            0: math.sqrt(7.0 / (16.0 * pi)) * (5.0 * nz * nz * nz - 3.0 * nz),
            1: math.sqrt(21.0 / (32.0 * pi)) * nx * (5.0 * nz * nz - 1.0),
            2: math.sqrt(105.0 / (16.0 * pi)) * (nx * nx - ny * ny) * nz,
            3: math.sqrt(35.0 / (32.0 * pi)) * (nx * nx - 3.0 * ny * ny) * nx,
        }.get(m, 0.0 * nx)
    elif l == 4:
        nz2, nx2, ny2 = nz * nz, nx * nx, ny * ny
        v = {
            -4: math.sqrt(315.0 / (256.0 * pi)) * 4.0 * nx * ny * (nx2 - ny2),
            -3: math.sqrt(315.0 / (32.0 * pi)) * ny * nz * (3.0 * nx2 - ny2),
            -2: math.sqrt(45.0 / (64.0 * pi)) * 2.0 * nx * ny * (7.0 * nz2 - 1.0),
            -1: math.sqrt(45.0 / (32.0 * pi)) * ny * nz * (7.0 * nz2 - 3.0),
            0: math.sqrt(9.0 / (256.0 * pi)) * (35.0 * nz2 * nz2 - 30.0 * nz2 + 3.0),
            1: math.sqrt(45.0 / (32.0 * pi)) * nx * nz * (7.0 * nz2 - 3.0),
            2: math.sqrt(45.0 / (64.0 * pi)) * (nx2 - ny2) * (7.0 * nz2 - 1.0),
            3: math.sqrt(315.0 / (32.0 * pi)) * nx * nz * (nx2 - 3.0 * ny2),
            4: math.sqrt(315.0 / (256.0 * pi)) * (nx2 * nx2 - 6.0 * nx2 * ny2 + ny2 * ny2),
        }.get(m, 0.0 * nx)
    else:
        v = 0.0 * nx
    v = np.asarray(v, dtype=np.float64) * np.ones_like(nx)
    if origin.any():
        v = np.where(origin, (1.0 / math.sqrt(4.0 * pi)) if l == 0 else 0.0, v)
    return v


# ---------------------------------------------------------------------------
# Synthetic UPF-shaped species
# ---------------------------------------------------------------------------


@dataclass
class Species:
    """UPF-shaped data of one species (fields the reference parser reads:
    src/features/pseudopotential/pseudopotential.zig:59-126)."""

    name: str
    z_val: float
    r: np.ndarray
    rab: np.ndarray
    vloc_r: np.ndarray  # Ry
    betas: list  # list of (l, r*beta(r))
    dij: np.ndarray  # [nbeta, nbeta], Ry
    gth: dict = field(default_factory=dict)

    @property
    def nbeta(self):
        return len(self.betas)

    @property
    def l_list(self):
        return [b[0] for b in self.betas]


# Builder-chosen parameters in the Goedecker-Teter-Hutter functional form
# (Phys. Rev. B 54, 1703 (1996)): V_loc(r) = -Z/r erf(r/(sqrt2 r_loc)) + exp(-(r/r_loc)^2/2) (C1 + C2 (r/r_loc)^2),
# projectors p_i^l(r) ~ r^(l+2(i-1)) exp(-r^2/(2 r_l^2)).  Energies below are Hartree.
SYNTHETIC_PARAMS = {
    "Si": dict(z=4.0, rloc=0.44, c1=-7.34, c2=0.0, chans=[(0, 0.423, [[5.9, 0.0], [0.0, 2.0]]), (1, 0.484, [[2.73]])]),
    "Al": dict(z=3.0, rloc=0.45, c1=-8.5, c2=0.0, chans=[(0, 0.46, [[5.1, 0.0], [0.0, 1.2]]), (1, 0.54, [[2.2]])]),
    "Ge": dict(z=4.0, rloc=0.54, c1=0.0, c2=0.0, chans=[(0, 0.42, [[7.5, 0.0], [0.0, 2.4]]), (1, 0.56, [[2.5]])]),
}


def _gth_projector(l: int, i: int, rl: float, r: np.ndarray) -> np.ndarray:
    """Normalised GTH projector p_i^l(r) (i = 1, 2, ...)."""
    e = l + (4.0 * i - 1.0) / 2.0
    return math.sqrt(2.0) * r ** (l + 2 * (i - 1)) * np.exp(-(r * r) / (2.0 * rl * rl)) / (rl**e * math.sqrt(math.gamma(e)))


def radial_mesh(z_mesh: float = 14.0, xmin: float = -7.0, dx: float = 0.0125, rmax: float = 10.0):
    """Logarithmic UPF-style mesh r_i = exp(xmin + i dx)/z with rab_i = r_i dx."""
    n = int((math.log(z_mesh * rmax) - xmin) / dx) + 1
    i = np.arange(n, dtype=np.float64)
    r = np.exp(xmin + i * dx) / z_mesh
    return r, r * dx


def synthetic_species(name: str) -> Species:
    p = SYNTHETIC_PARAMS[name]
    r, rab = radial_mesh()
    rloc = p["rloc"]
    from scipy.special import erf

    vloc_ha = -p["z"] / r * erf(r / (math.sqrt(2.0) * rloc)) + np.exp(-0.5 * (r / rloc) ** 2) * (
        p["c1"] + p["c2"] * (r / rloc) ** 2
    )
    betas = []
    blocks = []
    for l, rl, h in p["chans"]:
        h = np.asarray(h, dtype=np.float64)
        for i in range(h.shape[0]):
            betas.append((l, r * _gth_projector(l, i + 1, rl, r)))  # UPF stores r*beta(r)
        blocks.append(h)
    nb = len(betas)
    dij = np.zeros((nb, nb))
    off = 0
    for h in blocks:
        k = h.shape[0]
        dij[off : off + k, off : off + k] = 2.0 * h  # Hartree -> Ry
        off += k
    return Species(name=name, z_val=p["z"], r=r, rab=rab, vloc_r=2.0 * vloc_ha, betas=betas, dij=dij, gth=p)


def radial_tables(sp: Species, ecut_ry: float, n_points: int = 2048):
    """RadialTableSet.init (nonlocal.zig:312-338) with g_max from scf/common.zig:124-149."""
    g_max = 1.5 * math.sqrt(2.0 * ecut_ry)
    return [RadialTable(beta, sp.r, sp.rab, l, g_max, n_points) for (l, beta) in sp.betas]


@dataclass
class NonlocalSpecies:
    """nonlocal_context.zig:9-41 for a norm-conserving species."""

    species_index: int
    l_list: list
    m_offsets: list
    m_counts: list
    m_total: int
    dij: np.ndarray  # [nbeta, nbeta]
    phi: np.ndarray  # [m_total, n_pw] row-major

    @property
    def beta_count(self):
        return len(self.l_list)


def build_nonlocal_species(species_index: int, sp: Species, kpg: np.ndarray, tables=None) -> NonlocalSpecies:
    """nonlocal_context.zig:387-477 + fill_nonlocal_phi 524-549: phi = 4*pi*R_b(|k+G|)*Y_lm(k+G)."""
    l_list, m_offsets, m_counts = [], [], []
    total_m = 0
    gmag = np.sqrt(kpg[:, 0] ** 2 + kpg[:, 1] ** 2 + kpg[:, 2] ** 2)
    radial = []
    for b, (l, beta) in enumerate(sp.betas):
        l_list.append(l)
        m_offsets.append(total_m)
        m_counts.append(2 * l + 1)
        total_m += 2 * l + 1
        if tables is not None:
            radial.append(tables[b].eval(gmag))
        else:
            radial.append(np.array([radial_projector(beta, sp.r, sp.rab, l, float(g)) for g in gmag]))
    phi = np.zeros((total_m, kpg.shape[0]))
    for b, l in enumerate(l_list):
        for mi in range(2 * l + 1):
            m = mi - l
            ylm = real_ylm(l, m, kpg[:, 0], kpg[:, 1], kpg[:, 2])
            phi[m_offsets[b] + mi] = 4.0 * math.pi * radial[b] * ylm
    return NonlocalSpecies(species_index, l_list, m_offsets, m_counts, total_m, sp.dij.copy(), phi)


def expand_dij_m(ns: NonlocalSpecies) -> np.ndarray:
    """The radial D_ij applied per m (apply.zig:1186-1226) written as a dense m_total x m_total matrix:
    D_m[(b,m),(j,m)] = D_bj when l_b == l_j, else 0.  Equivalent to batch_apply_dij_radial."""
    mt = ns.m_total
    d = np.zeros((mt, mt))
    for b in range(ns.beta_count):
        for j in range(ns.beta_count):
            if ns.l_list[b] != ns.l_list[j]:
                continue
            for mi in range(ns.m_counts[b]):
                d[ns.m_offsets[b] + mi, ns.m_offsets[j] + mi] = ns.dij[b, j]
    return d


# -- local form factor (radial quadrature) ------------------------------------------------------


def local_vq_short_range(r: np.ndarray, rab: np.ndarray, vloc: np.ndarray, z_val: float, q: float) -> float:
    """form_factor.zig:223-262 (the default local_potential mode, config/defaults.zig:28):
    V(q) = 4 pi sum_i r_i^2 [V_loc(r_i) + 2 Z / r_i] sinc(q r_i) rab_i w_i - 8 pi Z / q^2 (Ry), the
    Coulomb term skipped at r < 1e-10 and at q < 1e-10 (where the short-range part alone is returned:
    compute_epsatm, form_factor.zig:264-268)."""
    n = r.size
    w = ctrap_weights(n)
    vc = np.where(r < 1e-10, 0.0, 2.0 * z_val / np.where(r < 1e-10, 1.0, r))
    x = q * r
    sinc = np.where(np.abs(x) < 1e-12, 1.0, np.sin(x) / np.where(np.abs(x) < 1e-12, 1.0, x))
    total = 0.0
    terms = r * r * (vloc + vc) * sinc * rab * w
    for t in terms:  # sequential sum, as the reference's loop
        total += t
    v = 4.0 * math.pi * total
    if q < 1e-10:
        return v
    return v - 8.0 * math.pi * z_val / (q * q)


def local_vq_short_range_vec(r, rab, vloc, z_val, q: np.ndarray) -> np.ndarray:
    """local_vq_short_range at many q at once (the sum over the mesh as a dot product)."""
    n = r.size
    w = ctrap_weights(n)
    vc = np.where(r < 1e-10, 0.0, 2.0 * z_val / np.where(r < 1e-10, 1.0, r))
    terms = r * r * (vloc + vc) * rab * w
    q = np.asarray(q, dtype=np.float64)
    x = np.outer(q, r)
    small = np.abs(x) < 1e-12
    sinc = np.where(small, 1.0, np.sin(x) / np.where(small, 1.0, x))
    v = 4.0 * math.pi * (sinc @ terms)
    big = q >= 1e-10
    v[big] -= 8.0 * math.pi * z_val / (q[big] * q[big])
    return v


def ionic_potential_radial(meshes, atom_species, positions, dims, recip, volume, g2max=0.0):
    """build_ionic_potential_grid (scf/potential.zig:279-318) with ionic_local_potential
    (hamiltonian.zig) and the short-range form factor: V(G) = (1 / Omega) sum_atoms V_s(|G|) e^{-i G tau}
    on the FFT-order box, 0 at |G| < 1e-10 and, with g2max > 0, for |G|^2 >= g2max.  meshes: per
    species (r, rab, vloc_Ry, z_valence)."""
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    gv = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ np.asarray(recip)
    g2 = (gv * gv).sum(axis=1)
    q = np.sqrt(g2)
    uq, inv = np.unique(q, return_inverse=True)
    vq = [local_vq_short_range_vec(m[0], m[1], m[2], m[3], uq)[inv] for m in meshes]
    vg = np.zeros(g2.size, complex)
    for a, s in enumerate(atom_species):
        vg += vq[s] * np.exp(-1j * (gv @ np.asarray(positions[a])))
    vg /= volume
    vg[q < 1e-10] = 0.0
    if g2max > 0.0:
        vg[g2 >= g2max] = 0.0
    return vg, vq
