"""Test infrastructure: the CPU restatement of the reference's nonlocal (Kleinman-Bylander) stress,
the oracle a device stress kernel is checked against, and the strained nonlocal energy it is the
derivative of.  Only tests use this module.  Ry units; stress in Ry/bohr^3.

  nonlocal_stress  src/features/stress/nonlocal_stress.zig:108-558 (project_p_and_dp,
                   compute_dp_bm, accumulate_nonlocal_sigma_for_band, compute_enl_for_band,
                   process_nonlocal_stress_band), norm-conserving projectors (no PAW q_ij)
  d_ylm_dq         src/features/stress/stress.zig:79-137 (l <= 2, analytic)

The reference accumulates only the components a <= b (accumulate_nonlocal_sigma_for_band loops
b over a..2) and leaves the lower triangle zero; the restatement does the same.
"""
from __future__ import annotations

import math

import numpy as np

from oracle.pseudo import real_ylm


def d_ylm_dq(l, m, q):
    """Gradient of Y_lm(q / |q|) with respect to q (n rows, 3): (grad_n Y - n (n . grad_n Y)) / |q|,
    zero at |q| < 1e-15 and for l = 0."""
    q = np.asarray(q, dtype=np.float64)
    qm = np.sqrt((q * q).sum(axis=1))
    out = np.zeros_like(q)
    if l == 0:
        return out
    ok = qm >= 1e-15
    inv = np.where(ok, 1.0 / np.where(ok, qm, 1.0), 0.0)
    n = q * inv[:, None]
    nx, ny, nz = n[:, 0], n[:, 1], n[:, 2]
    z = np.zeros_like(nx)
    if l == 1:
        c = math.sqrt(3.0 / (4.0 * math.pi))
        g = {-1: (z, z + c, z), 0: (z, z, z + c), 1: (z + c, z, z)}[m]
    elif l == 2:
        c0 = math.sqrt(5.0 / (16.0 * math.pi))
        c1 = math.sqrt(15.0 / (4.0 * math.pi))
        c2 = math.sqrt(15.0 / (16.0 * math.pi))
        g = {-2: (2 * c2 * ny, 2 * c2 * nx, z), -1: (z, c1 * nz, c1 * ny), 0: (z, z, 6 * c0 * nz),
             1: (c1 * nz, z, c1 * nx), 2: (2 * c2 * nx, -2 * c2 * ny, z)}[m]
    else:
        raise NotImplementedError("d_ylm_dq: l <= 2")
    g = np.stack(g, axis=1)
    ndg = (n * g).sum(axis=1)
    return (g - n * ndg[:, None]) * inv[:, None]


def _offsets(l_list):
    offs, tot = [], 0
    for l in l_list:
        offs.append(tot)
        tot += 2 * l + 1
    return offs, tot


def _dp(l_list, dij, p):
    """Dp_bm = sum_j D_bj p_jm over channels j of the same l (compute_dp_bm)."""
    offs, _ = _offsets(l_list)
    dp = np.zeros_like(p)
    for b, lb in enumerate(l_list):
        for j, lj in enumerate(l_list):
            if lj != lb or dij[b, j] == 0.0:
                continue
            for m in range(2 * lb + 1):
                dp[offs[b] + m] += dij[b, j] * p[offs[j] + m]
    return dp


def projector_derivatives(l_list, rad, drad, kpg):
    """phi_bm(q) = 4 pi R_b(|q|) Y_lm(q) (m_total, n) and dphi_bm/dq_a = 4 pi (R_b' n_a Y_lm +
    R_b dY_lm/dq_a) (m_total, 3, n), zero where |q| < 1e-12 (project_p_and_dp,
    nonlocal_stress.zig:108-165); rad(b, q), drad(b, q) give R_b and R_b'."""
    kpg = np.asarray(kpg, dtype=np.float64)
    qm = np.sqrt((kpg * kpg).sum(axis=1))
    live = qm >= 1e-12
    inv = np.where(live, 1.0 / np.where(live, qm, 1.0), 0.0)
    nhat = kpg * inv[:, None]
    offs, mt = _offsets(l_list)
    phi = np.zeros((mt, len(kpg)))
    dphi = np.zeros((mt, 3, len(kpg)))
    for b, l in enumerate(l_list):
        r, dr = rad(b, qm), drad(b, qm)
        for mi in range(2 * l + 1):
            m = mi - l
            y = real_ylm(l, m, kpg[:, 0], kpg[:, 1], kpg[:, 2])
            dy = d_ylm_dq(l, m, kpg)
            phi[offs[b] + mi] = 4.0 * math.pi * r * y
            dphi[offs[b] + mi] = 4.0 * math.pi * (dr[None, :] * nhat.T * y[None, :] + r[None, :] * dy.T) * live[None, :]
    return phi, dphi


def nonlocal_stress(kpg, gcart, species, atom_species, positions, vectors, weights, volume):
    """sigma_ab (a <= b) = -(2 f_n / Omega^2) sum_G sum_bm dphi_bm/dq_a q_b Re[conj(Dp_bm) S(G) c(G)]
    - delta_ab f_n E_nl,n / Omega over bands n and atoms, with p_bm = sum_G phi_bm(G) S(G) c(G),
    phi_bm = 4 pi R_b(|q|) Y_lm(q), S(G) = e^{i G . tau} (G without k, as the reference),
    E_nl,n = Re sum_bm conj(p_bm) Dp_bm / Omega, q = k + G.
    species: per species (l_list, D (nb x nb, Ry), R(b, q), dR/dq(b, q)); weights: f_n = occupation x
    k weight x spin factor per band (bands with f_n <= 0 are skipped)."""
    kpg = np.asarray(kpg, dtype=np.float64)
    gcart = np.asarray(gcart, dtype=np.float64)
    sigma = np.zeros((3, 3))
    vecs = np.asarray(vectors)
    for s, tau in zip(atom_species, np.asarray(positions, dtype=np.float64)):
        l_list, dij, rad, drad = species[s]
        dij = np.asarray(dij, dtype=np.float64)
        phi, dphi = projector_derivatives(l_list, rad, drad, kpg)
        phase = np.exp(1j * (gcart @ tau))
        for f, c in zip(weights, vecs):
            if f <= 0.0:
                continue
            pc = phase * c
            p = phi @ pc
            dp = _dp(l_list, dij, p)
            z = np.real(np.conj(dp)[:, None] * pc[None, :])  # (mt, G)
            pref = 2.0 * f / volume**2
            for a in range(3):
                t = (dphi[:, a, :] * z).sum(axis=0)  # per G
                for b in range(a, 3):
                    sigma[a, b] -= pref * float((t * kpg[:, b]).sum())
            e_nl = float(np.real(np.conj(p) @ dp)) / volume
            for a in range(3):
                sigma[a, a] += -f * e_nl / volume
    return sigma


def nonlocal_energy(kpg, gcart, species, atom_species, positions, vectors, weights, volume, strain=None):
    """sum_n f_n sum_atoms Re sum_bm conj(p_bm) Dp_bm / Omega, optionally for the homogeneously
    deformed cell x -> (I + strain) x at fixed plane-wave coefficients: q -> (I + strain)^-T q,
    Omega -> Omega det(I + strain), G . tau unchanged."""
    kpg = np.asarray(kpg, dtype=np.float64)
    F = np.eye(3) + (np.zeros((3, 3)) if strain is None else np.asarray(strain, dtype=np.float64))
    q = kpg @ np.linalg.inv(F)  # rows: (F^-T q)^T = q^T F^-1
    vol = volume * float(np.linalg.det(F))
    qm = np.sqrt((q * q).sum(axis=1))
    e = 0.0
    vecs = np.asarray(vectors)
    for s, tau in zip(atom_species, np.asarray(positions, dtype=np.float64)):
        l_list, dij, rad, _ = species[s]
        dij = np.asarray(dij, dtype=np.float64)
        offs, mt = _offsets(l_list)
        phi = np.zeros((mt, len(q)))
        for b, l in enumerate(l_list):
            r = rad(b, qm)
            for mi in range(2 * l + 1):
                phi[offs[b] + mi] = 4.0 * math.pi * r * real_ylm(l, mi - l, q[:, 0], q[:, 1], q[:, 2])
        phase = np.exp(1j * (np.asarray(gcart, dtype=np.float64) @ tau))
        for f, c in zip(weights, vecs):
            if f <= 0.0:
                continue
            p = phi @ (phase * c)
            e += f * float(np.real(np.conj(p) @ _dp(l_list, dij, p))) / vol
    return e
