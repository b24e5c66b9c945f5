"""Test infrastructure: the CPU restatement of the Hellmann-Feynman forces that the device force
entry points (dftcuda_local_forces, dftcuda_nonlocal_forces) and the host Ewald forces are checked
against.  Only tests use it.  Forces in Ry/bohr, positions Cartesian bohr."""
from __future__ import annotations

import math

import numpy as np

from oracle import potential as op


def local_forces(rho, gth, atom_species, positions, dims, recip, g2max=0.0):
    """local_pseudo_forces (forces/local_force.zig:21-80): F_a = sum_G 2 ff_s(|G|) G Im(e^{iG.tau_a}
    rho(G)) over 1e-12 < G^2 <= g2max, with rho(G) = (1/N) sum_r rho e^{-iGr} and ff the GTH local
    form factor (Hartree; x2 for Ry)."""
    gth = np.asarray(gth, dtype=np.float64).reshape(-1, 6)
    G = op.g_vectors_cart(dims, recip)
    g2 = (G * G).sum(axis=1)
    keep = g2 > 1e-12
    if g2max > 0.0:
        keep &= g2 <= g2max
    G, g2 = G[keep], g2[keep]
    rg = op.to_g(rho, dims)[keep]
    out = np.zeros((len(atom_species), 3))
    for a, (s, tau) in enumerate(zip(atom_species, np.asarray(positions, dtype=np.float64))):
        Z, r, c1, c2, c3, c4 = gth[s]
        y = g2 * r * r
        e = np.exp(-0.5 * y)
        poly = c1 + c2 * (3 - y) + c3 * (15 - 10 * y + y * y) + c4 * (105 - 105 * y + 21 * y * y - y ** 3)
        ff = -4 * math.pi * Z / g2 * e + math.sqrt(8 * math.pi ** 3) * r ** 3 * e * poly
        w = 2.0 * ff * np.imag(np.exp(1j * (G @ tau)) * rg)
        out[a] = (G * w[:, None]).sum(axis=0)
    return out


def nonlocal_forces(kpg, species_phi, atom_species, positions, vectors, weights, volume):
    """accumulate_atom_force_at_kpoint / accumulate_band_force (forces/nonlocal_force.zig:283-386)
    for norm-conserving Kleinman-Bylander projectors: per atom, phase(G) = e^{+i(k+G).R},
    p_bm = sum_G phi_bm(G) phase(G) c(G), Dp = D p (same l), q(G) = sum_bm conj(Dp_bm) phi_bm(G),
    F += (2 w_b / vol) sum_G (k+G) Im[q(G) phase(G) c(G)].
    kpg: (n, 3) Cartesian k+G; species_phi: per species (l_list, D (nb x nb), phi (m_total, n));
    vectors: (nbands, n); weights: k weight x occupation x spin per band."""
    kpg = np.asarray(kpg, dtype=np.float64)
    out = np.zeros((len(atom_species), 3))
    vecs = np.asarray(vectors)
    for a, (s, tau) in enumerate(zip(atom_species, np.asarray(positions, dtype=np.float64))):
        l_list, dij, phi = species_phi[s]
        phi = np.asarray(phi, dtype=np.float64)
        dij = np.asarray(dij, dtype=np.float64)
        offs, tot = [], 0
        for l in l_list:
            offs.append(tot)
            tot += 2 * l + 1
        phase = np.exp(1j * (kpg @ tau))
        for bnd, w in enumerate(weights):
            if w <= 0.0:
                continue
            c = vecs[bnd]
            p = phi @ (phase * c)  # (m_total,)
            dp = np.zeros_like(p)
            for i, li in enumerate(l_list):
                for j, lj in enumerate(l_list):
                    if li != lj or dij[i, j] == 0.0:
                        continue
                    for m in range(2 * li + 1):
                        dp[offs[i] + m] += dij[i, j] * p[offs[j] + m]
            q = np.conj(dp) @ phi  # (n,)
            z = q * phase * c
            out[a] += 2.0 * w / volume * (kpg * np.imag(z)[:, None]).sum(axis=0)
    return out


def ewald_forces(cell, charges, positions, eta, tol=1e-14):
    """Ion-ion forces (compute_ion_ion_forces, forces/forces.zig:59-104): minus the derivative of
    the Ewald energy (real-space erfc sum and reciprocal sum), in Ry/bohr."""
    from scipy.special import erfc

    cell = np.asarray(cell, dtype=np.float64)
    pos = np.asarray(positions, dtype=np.float64)
    z = np.asarray(charges, dtype=np.float64)
    vol = abs(np.linalg.det(cell))
    recip = 2.0 * math.pi * np.linalg.inv(cell).T
    rcut = math.sqrt(-math.log(tol)) / eta + 1e-9
    gcut = 2.0 * eta * math.sqrt(-math.log(tol))
    na = [int(math.ceil(rcut * np.linalg.norm(recip[i]) / (2.0 * math.pi))) + 1 for i in range(3)]
    rng = [np.arange(-n, n + 1) for n in na]
    L = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ cell
    out = np.zeros_like(pos)
    for i in range(len(z)):
        d = pos[i][None, None, :] - pos[:, None, :] + L[None, :, :]  # [j, L, 3]
        r = np.linalg.norm(d, axis=2)
        m = (r > 1e-10) & (r < rcut)
        rr = np.where(m, r, 1.0)
        g = (erfc(eta * rr) / rr**2 + 2.0 * eta / math.sqrt(math.pi) * np.exp(-eta * eta * rr * rr) / rr) / rr
        out[i] += z[i] * ((z[:, None] * np.where(m, g, 0.0))[:, :, None] * d).sum(axis=(0, 1))
    ng = [int(math.ceil(gcut / np.linalg.norm(recip[i]))) + 1 for i in range(3)]
    rng = [np.arange(-n, n + 1) for n in ng]
    G = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ recip
    g2 = (G * G).sum(axis=1)
    sel = (g2 > 1e-12) & (g2 < gcut * gcut)
    G, g2 = G[sel], g2[sel]
    S = np.exp(1j * (G @ pos.T)) @ z
    k = np.exp(-g2 / (4.0 * eta * eta)) / g2
    for i in range(len(z)):
        out[i] += (4.0 * math.pi / vol) * z[i] * (G * (k * np.imag(np.exp(1j * (G @ pos[i])) * np.conj(S)))[:, None]).sum(axis=0)
    return 2.0 * out


def local_forces_radial(rho, meshes, atom_species, positions, dims, recip, g2max=0.0):
    """local_pseudo_forces (forces/local_force.zig:66-111) with the short-range form factor of each
    species' radial mesh (pseudo.local_vq_short_range, form_factor.zig:223-262): F_a = sum_G V_s(|G|) G
    Im(e^{iG.tau_a} rho(G)) over |G| >= 1e-10 and G^2 < g2max.  meshes: (r, rab, vloc_Ry, z) per species."""
    from oracle import pseudo

    G = op.g_vectors_cart(dims, recip)
    g2 = (G * G).sum(axis=1)
    q = np.sqrt(g2)
    keep = q >= 1e-10
    if g2max > 0.0:
        keep &= g2 < g2max
    G, q = G[keep], q[keep]
    rg = op.to_g(rho, dims)[keep]
    uq, inv = np.unique(q, return_inverse=True)
    vq = [pseudo.local_vq_short_range_vec(m[0], m[1], m[2], m[3], uq)[inv] for m in meshes]
    out = np.zeros((len(atom_species), 3))
    for a, (s, tau) in enumerate(zip(atom_species, np.asarray(positions, dtype=np.float64))):
        w = vq[s] * np.imag(np.exp(1j * (G @ tau)) * rg)
        out[a] = (G * w[:, None]).sum(axis=0)
    return out
