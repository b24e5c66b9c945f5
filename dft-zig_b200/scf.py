"""Host-side SCF driver around the GPU hot path (the caller's side of the boundary).

dft-zig keeps its SCF driver in Zig; this module restates the pieces needed to reach total energies
and time-to-SCF with the hot path on the GPU, each following the cited reference code:

  flat start rho_0 = N_e / Omega                  scf/run_state.zig:98-115
  V_H(G) = 8 pi rho(G) / |G|^2 (Ry)               scf/potential.zig:34-41
  LDA-PZ exchange-correlation (Ry)                xc/xc.zig:195-211, 344-384
  V = V_ion + V_H + V_xc, real part on the grid   scf/potential.zig:144-203, 320-334
  potential mixing (linear, then Pulay/DIIS from pulay_start on V_Hxc)
                                                  scf/scf.zig:148-188, scf/mixing.zig:182-248
  convergence on RMS(rho_out - rho_in)            scf/scf.zig:392-410, scf/util.zig:17-24
  fixed occupations / Fermi-Dirac + Fermi level   kpoint/density.zig:98-112, scf/fermi_level.zig
  total energy = band + (-E_H - int V_xc rho + E_xc) + E_ion-ion + psp_core - TS
                                                  scf/energy.zig:372-396
  Ewald ion-ion energy                            ewald/ewald.zig (standard Ewald split)
  eigensolver warm start from the previous iteration's vectors
                                                  kpoint/data.zig:7-46, defaults.zig:40
  warm-up iterations with looser eigensolver settings
                                                  scf/density.zig:167-176, defaults.zig:37-39

The hot path (H|psi>, the Davidson solver, the band density) runs through a backend object:
``GpuBackend`` drives libdftcuda through the package's KpointContext.  Tests plug in other
backends through the same small interface.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import kpar
from . import system as sysm


# ---------------------------------------------------------------------------------------------
# Exchange-correlation, Hartree, ionic terms
# ---------------------------------------------------------------------------------------------


def lda_pz(n: np.ndarray):
    """xc.zig:195-211, 344-384: returns (f, v) in Ry (f per unit volume, v = df/dn); n <= 1e-12 -> 0."""
    n = np.asarray(n, dtype=np.float64)
    f = np.zeros_like(n)
    v = np.zeros_like(n)
    m = n > 1e-12
    nn = n[m]
    n13 = np.power(nn, 1.0 / 3.0)
    c_x = -0.75 * (3.0 / math.pi) ** (1.0 / 3.0)
    ex = nn * c_x * n13
    rs = np.power(3.0 / (4.0 * math.pi * nn), 1.0 / 3.0)
    eps_c = np.empty_like(nn)
    v_c = np.empty_like(nn)
    lo = rs < 1.0
    a, b, c, d = 0.0311, -0.048, 0.0020, -0.0116
    r = rs[lo]
    lr = np.log(r)
    e = a * lr + b + c * r * lr + d * r
    de = a / r + c * lr + c + d
    eps_c[lo] = e
    v_c[lo] = e - (r / 3.0) * de
    g, b1, b2 = -0.1423, 1.0529, 0.3334
    r = rs[~lo]
    sr = np.sqrt(r)
    den = 1.0 + b1 * sr + b2 * r
    e = g / den
    de = -g * (0.5 * b1 / sr + b2) / (den * den)
    eps_c[~lo] = e
    v_c[~lo] = e - (r / 3.0) * de
    f[m] = 2.0 * (ex + nn * eps_c)
    v[m] = 2.0 * (4.0 / 3.0 * c_x * n13 + v_c)
    return f, v


def ewald_energy(cell: np.ndarray, charges: np.ndarray, pos: np.ndarray, tol: float = 1e-14, eta: Optional[float] = None) -> float:
    """Ion-ion energy (Ry) by the Ewald split: real-space erfc sum + reciprocal sum - self - background.
    The split parameter eta (bohr^-1) does not change the result; by default it follows the atom
    density, 0.85 sqrt(pi) (N / V^2)^(1/6), which balances the real-space image sum against the
    reciprocal one for large cells (Si216: 0.3 s instead of seconds)."""
    from scipy.special import erfc

    vol = abs(np.linalg.det(cell))
    recip = 2.0 * math.pi * np.linalg.inv(cell).T
    if eta is None:
        eta = 0.85 * math.sqrt(math.pi) * (len(charges) / vol**2) ** (1.0 / 6.0)
    # real-space cutoff where erfc(eta r) < tol, reciprocal cutoff where exp(-G^2/4eta^2) < tol
    rcut = math.sqrt(-math.log(tol)) / eta + 1e-9
    gcut = 2.0 * eta * math.sqrt(-math.log(tol))
    na = [int(math.ceil(rcut * np.linalg.norm(recip[i]) / (2.0 * math.pi))) + 1 for i in range(3)]
    e_real = 0.0
    rng = [np.arange(-n, n + 1) for n in na]
    L = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ cell
    dmax = float(np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=2).max())
    L = L[np.linalg.norm(L, axis=1) < rcut + dmax + 1e-9]  # |d + L| < rcut needs |L| < rcut + |d|
    for i in range(len(charges)):
        d = pos[i][None, :] - pos  # [j, 3]
        r = np.linalg.norm(d[:, None, :] + L[None, :, :], axis=2)  # [j, L]
        mask = (r > 1e-10) & (r < rcut)
        rr = r[mask]
        e_real += 0.5 * charges[i] * float(np.sum(np.broadcast_to(charges[:, None], r.shape)[mask] * erfc(eta * rr) / rr))
    ng = [int(math.ceil(gcut / np.linalg.norm(recip[i]))) + 1 for i in range(3)]
    rng = [np.arange(-n, n + 1) for n in ng]
    G = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ recip
    g2 = (G * G).sum(axis=1)
    sel = (g2 > 1e-12) & (g2 < gcut * gcut)
    G, g2 = G[sel], g2[sel]
    sf = np.exp(1j * (G @ pos.T)) @ charges
    e_rec = (2.0 * math.pi / vol) * np.sum(np.abs(sf) ** 2 * np.exp(-g2 / (4.0 * eta * eta)) / g2)
    e_self = -eta / math.sqrt(math.pi) * np.sum(charges**2)
    e_bg = -math.pi * np.sum(charges) ** 2 / (2.0 * eta * eta * vol)
    return 2.0 * float(e_real + e_rec + e_self + e_bg)


def ewald_forces(cell: np.ndarray, charges: np.ndarray, pos: np.ndarray, tol: float = 1e-14, eta: Optional[float] = None) -> np.ndarray:
    """Ion-ion forces (Ry/bohr; compute_ion_ion_forces, forces/forces.zig:59-104): minus the
    gradient of ewald_energy, real-space erfc sum and reciprocal sum with the same split."""
    from scipy.special import erfc

    pos = np.asarray(pos, dtype=np.float64)
    charges = np.asarray(charges, dtype=np.float64)
    vol = abs(np.linalg.det(cell))
    recip = 2.0 * math.pi * np.linalg.inv(cell).T
    if eta is None:
        eta = 0.85 * math.sqrt(math.pi) * (len(charges) / vol**2) ** (1.0 / 6.0)
    rcut = math.sqrt(-math.log(tol)) / eta + 1e-9
    gcut = 2.0 * eta * math.sqrt(-math.log(tol))
    na = [int(math.ceil(rcut * np.linalg.norm(recip[i]) / (2.0 * math.pi))) + 1 for i in range(3)]
    rng = [np.arange(-n, n + 1) for n in na]
    L = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ cell
    dmax = float(np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=2).max())
    L = L[np.linalg.norm(L, axis=1) < rcut + dmax + 1e-9]
    f = np.zeros_like(pos)
    c2 = 2.0 * eta / math.sqrt(math.pi)
    for i in range(len(charges)):
        d = pos[i][None, None, :] - pos[:, None, :] + L[None, :, :]  # [j, L, 3]
        r = np.linalg.norm(d, axis=2)
        m = (r > 1e-10) & (r < rcut)
        rr = np.where(m, r, 1.0)
        radial = np.where(m, (erfc(eta * rr) / rr + c2 * np.exp(-(eta * rr) ** 2)) / (rr * rr), 0.0)
        f[i] += charges[i] * np.einsum("jl,jlx->x", charges[:, None] * radial, d)
    ng = [int(math.ceil(gcut / np.linalg.norm(recip[i]))) + 1 for i in range(3)]
    rng = [np.arange(-n, n + 1) for n in ng]
    G = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) @ recip
    g2 = (G * G).sum(axis=1)
    sel = (g2 > 1e-12) & (g2 < gcut * gcut)
    G, g2 = G[sel], g2[sel]
    ph = np.exp(1j * (G @ pos.T))  # [G, atom]
    S = ph @ charges
    k = np.exp(-g2 / (4.0 * eta * eta)) / g2
    f += (4.0 * math.pi / vol) * charges[:, None] * (np.imag(ph * np.conj(S)[:, None]) * k[:, None]).T @ G
    return 2.0 * f


# ---------------------------------------------------------------------------------------------
# Mixing
# ---------------------------------------------------------------------------------------------


def _solve_pulay_system(B, rhs):
    """mixing.zig:341-405: Gaussian elimination with partial pivoting of the bordered system, the
    overlap block first divided by its largest diagonal entry (the weights do not change).  Returns
    None for a pivot below 1e-12 (the reference averages the history then; the mixer drops its
    oldest pair and solves again instead, which keeps DIIS working once more pairs are held than
    the residuals have independent directions)."""
    A = np.array(B, dtype=np.float64)
    m = A.shape[0] - 1
    d = float(np.max(np.diag(A)[:m]))
    if d > 0.0:
        A[:m, :m] /= d
    b = np.array(rhs, dtype=np.float64)
    size = b.size
    for col in range(size):
        max_row = col + int(np.argmax(np.abs(A[col:, col])))
        if max_row != col:
            A[[col, max_row]] = A[[max_row, col]]
            b[[col, max_row]] = b[[max_row, col]]
        pivot = A[col, col]
        if abs(pivot) < 1e-12:
            return None
        for row in range(col + 1, size):
            f = A[row, col] / pivot
            A[row, col:] -= f * A[col, col:]
            b[row] -= f * b[col]
    r = np.zeros(size)
    for i in range(size - 1, -1, -1):
        r[i] = (b[i] - np.dot(A[i, i + 1:], r[i + 1:])) / A[i, i]
    return r


class PulayMixer:
    """mixing.zig:182-248 (mix_with_residual): history of inputs and residuals, DIIS coefficients
    from B_ij = <R_i|R_j> with the constraint sum c = 1, new = sum c_i (x_i + beta R_i); a singular
    system drops the oldest pairs (see _solve_pulay_system)."""

    def __init__(self, history: int):
        self.history = history
        self.xs: list = []
        self.rs: list = []

    def mix(self, x: np.ndarray, residual: np.ndarray, beta: float) -> np.ndarray:
        self.xs.append(x.copy())
        self.rs.append(residual.copy())
        while len(self.xs) > self.history:
            self.xs.pop(0)
            self.rs.pop(0)
        m = len(self.xs)
        first = 0  # oldest pair used
        c = None
        while m - first >= 2:
            k = m - first
            B = np.zeros((k + 1, k + 1))
            for i in range(k):
                for j in range(k):
                    B[i, j] = float(np.dot(self.rs[first + i], self.rs[first + j]))
            B[:k, k] = -1.0
            B[k, :k] = -1.0
            rhs = np.zeros(k + 1)
            rhs[k] = -1.0
            c = _solve_pulay_system(B, rhs)
            if c is not None:
                break
            first += 1
        if c is None:
            return x + beta * residual
        out = np.zeros_like(x)
        for i in range(m - first):
            out += c[i] * (self.xs[first + i] + beta * self.rs[first + i])
        return out


# ---------------------------------------------------------------------------------------------
# Occupations
# ---------------------------------------------------------------------------------------------


def fd_occ(e, mu, sigma):
    x = np.clip((np.asarray(e) - mu) / sigma, -700.0, 700.0)
    return 1.0 / (1.0 + np.exp(x))


def fermi_level(nelec, sigma, kweights, values, spin=2.0):
    """fermi_level.zig:61-124 (bracket with padding max(10 sigma, 1e-3), <= 80 bisections)."""
    allv = np.concatenate([np.asarray(v) for v in values])
    lo_e, hi_e = float(allv.min()), float(allv.max())

    def count(mu):
        return sum(spin * w * float(fd_occ(v, mu, sigma).sum()) for w, v in zip(kweights, values))

    pad = max(10.0 * sigma, 1e-3)
    low, high = lo_e - pad, hi_e + pad
    for _ in range(12):
        if count(low) <= nelec <= count(high):
            break
        pad *= 2.0
        low, high = lo_e - pad, hi_e + pad
    left, right = low, high
    for _ in range(80):
        mid = 0.5 * (left + right)
        c = count(mid)
        if abs(c - nelec) < 1e-8:
            return mid
        if c > nelec:
            right = mid
        else:
            left = mid
    return 0.5 * (left + right)


def entropy_term(occ):
    o = np.asarray(occ)
    m = (o > 1e-12) & (o < 1.0 - 1e-12)
    s = np.zeros_like(o)
    s[m] = -(o[m] * np.log(o[m]) + (1.0 - o[m]) * np.log(1.0 - o[m]))
    return s


# ---------------------------------------------------------------------------------------------
# Backend: the hot path on the GPU
# ---------------------------------------------------------------------------------------------


class GpuBackend:
    """One libdftcuda k-point context per k-point (the GPU analogue of KpointApplyCache).

    precision "fp64" runs every pass in FP64.  "mixed" keeps a second context per k-point in
    TF32X3 precision (FP32 FFT passes, split-TF32 tensor-core projector and Rayleigh-Ritz GEMMs) and
    uses it while the SCF density residual is above ``switch_drho`` (1e-4), then the FP64 one for the rest.
    It also switches when the residual stops falling near that threshold (``stall`` iterations below
    10 x switch_drho without a new minimum), the sign that the reduced-precision operator's error
    floor has been reached.  Orthonormalisation,
    the subspace eigensolver, residual checks, occupations and energies stay FP64 throughout."""

    def __init__(self, dz, precision="fp64", switch_drho: float = 1e-4, stall: int = 3, precond=None,
                 resident: bool = False, min_pw_reduced: int = 4096):
        self.dz = dz
        self.precision = precision
        # resident: eigenvectors stay on the device between iterations, and the SCF state (density,
        # Hartree-XC potential, Pulay history) lives there too (ScfState uses the device potential)
        self.resident = resident
        self.precond = precond  # None (reference form) or (kind, params) for every context
        self.switch_drho = switch_drho
        self.stall = stall
        self.ctxs = []
        self.ctxs32 = []
        self.use32 = precision == "mixed"
        self.local_r = None
        self.best = float("inf")
        self.since_best = 0
        self.switched_at = None
        self.n_obs = 0
        self.solves = []  # (precision, Davidson iterations, H applications) per eig_all call
        # mixed: k-points with fewer plane waves keep their FP64 context throughout; their solves are
        # bound by kernel issue, not by arithmetic or bytes, and a second context only adds launches
        # (Al4 at 25 Ry, ~950 plane waves: 8.0 s mixed against 5.5 s FP64 before this rule)
        self.min_pw_reduced = min_pw_reduced

    def _make(self, inp, prec):
        kc = self.dz.KpointContext(*inp.dims, inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, prec)
        kc.set_projectors([self.dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
        if self.precond is not None:
            kc.set_preconditioner(*self.precond)
        return kc

    def setup(self, kinputs):
        for inp in kinputs:
            self.ctxs.append(self._make(inp, 0))
            if self.precision == "mixed":
                small = inp.basis.n < self.min_pw_reduced
                self.ctxs32.append(self.ctxs[-1] if small else self._make(inp, self.dz.PRECISION_TF32X3))

    def observe(self, drho: float):
        self.n_obs += 1
        if drho < self.best:
            self.best, self.since_best = drho, 0
        elif drho < 10.0 * self.switch_drho:
            # a stall counts only near the switch threshold, where the reduced-precision floor lies;
            # above it a rising residual is the mixing's own transient (the FP64 run shows it too)
            self.since_best += 1
        if self.use32 and (drho < self.switch_drho or self.since_best >= self.stall):
            self.use32 = False
            self.switched_at = self.n_obs
            if self.local_r is not None:
                for kc in self.ctxs:
                    kc.set_vloc(self.local_r)

    def _active(self):
        return self.ctxs32 if self.use32 else self.ctxs

    def set_vloc(self, local_r):
        self.local_r = local_r
        for kc in self._active():
            kc.set_vloc(local_r)

    def eig(self, k, diag, nbands, opts: dict, init):
        o = self.dz.Options(**opts, init_vectors=init)
        r = self._active()[k].hermitian_eigen_decomp_iterative(diag, nbands, o)
        return r.values, r.vectors

    def eig_all(self, diags, nbands, opts: dict, inits):
        """All k-points in one lockstep batch (dftcuda_eig_solve_batch)."""
        rs = self.dz.hermitian_eigen_decomp_iterative_batch(self._active(), diags, nbands, self.dz.Options(**opts), inits,
                                                            device=self.resident)
        self.solves.append(("tf32x3" if self.use32 else "fp64", max(r.iterations for r in rs), sum(r.h_applies for r in rs)))
        return [(r.values, r.vectors) for r in rs]

    def density(self, k, vectors, weights, rho):
        self._active()[k].accumulate_band_density(vectors, weights, rho)

    def nonlocal_energies(self, k, vectors):
        return self._active()[k].nonlocal_energies(vectors)

    def nonlocal_forces(self, k, vectors, weights, natoms):
        return self._active()[k].nonlocal_forces(vectors, weights, natoms)

    def close(self):
        seen = set()
        for kc in self.ctxs + self.ctxs32:
            if id(kc) not in seen:
                seen.add(id(kc))
                kc.close()
        self.ctxs = []
        self.ctxs32 = []


# ---------------------------------------------------------------------------------------------
# The SCF loop
# ---------------------------------------------------------------------------------------------


@dataclass
class ScfParams:
    ecut: float
    kmesh: tuple
    nbands: int
    mixing_beta: float = 0.3
    pulay_history: int = 8
    pulay_start: int = 4
    max_iter: int = 50
    convergence: float = 1e-6
    iterative_max_iter: int = 20
    iterative_tol: float = 1e-4
    warmup_steps: int = 2
    warmup_max_iter: int = 10
    warmup_tol: float = 1e-3
    reuse_vectors: bool = True
    smearing: Optional[float] = None  # Fermi-Dirac width (Ry); None = fixed occupations
    xc: str = "lda"  # "lda" (LDA-PZ) or "pbe" (the resident driver's device potential)
    energy_tol_per_atom: Optional[float] = None  # stop once |E - E_target| < tol (time-to-SCF runs)
    energy_target: Optional[float] = None
    initial_density: Optional[np.ndarray] = None  # rho(r) on the FFT grid; None = flat N_e / Omega
    kpoints: Optional[list] = None  # explicit [(k_frac, weight)] in place of the kmesh (weights sum to 1)
    # model dielectric preconditioner of the Pulay residual (apply_model_dielectric_preconditioner,
    # scf/mixing.zig:319-337; off at diemac = 1, the reference default; its config validation
    # suggests ~12 for semiconductors at tight convergence)
    diemac: float = 1.0
    dielng: float = 1.0


@dataclass
class ScfResult:
    converged: bool
    iterations: int
    energy: float
    energy_per_atom: float
    eigenvalues: list
    terms: dict
    rho: np.ndarray
    history: list = field(default_factory=list)
    wall_s: float = 0.0
    forces: Optional[np.ndarray] = None  # (natoms, 3) Ry/bohr when run_scf(..., forces=True)


def g_vectors(dims, recip):
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    G = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ recip
    return (G * G).sum(axis=1)


def ionic_potential_g(c: sysm.Crystal, dims, ecut: float) -> np.ndarray:
    """V_ion(G) on the FFT grid (Ry), G = 0 term 0, |G|^2 <= 4 ecut (the same form factors as
    system.local_potential)."""
    n = dims[0] * dims[1] * dims[2]
    vr = sysm.local_potential(c, dims, ecut)
    return np.fft.fftn(vr.reshape(dims[2], dims[1], dims[0])).ravel() / n


class ScfState:
    """One cell's SCF loop (scf.zig:148-188 control flow) split around its eigensolves, so several
    cells can share one batched eigensolver call per iteration (run_scf_many)."""

    def __init__(self, c: sysm.Crystal, p: ScfParams, backend, verbose: bool = False, comm=None, table_cache=None):
        self.t0 = time.perf_counter()
        self.c, self.p, self.backend, self.verbose = c, p, backend, verbose
        self.comm = comm if comm is not None else kpar.SerialComm()
        dims = self.dims = sysm.fft_box(p.ecut, c.recip)
        N = self.N = dims[0] * dims[1] * dims[2]
        self.vol = c.volume
        kpts = [(np.asarray(k, float), float(w)) for k, w in p.kpoints] if p.kpoints is not None else sysm.monkhorst_pack(p.kmesh)
        self.nk = len(kpts)
        # k-points dealt to the ranks by basis size; this rank builds inputs and contexts for its own
        costs = [sysm.basis(c.recip, p.ecut, k).hkl.shape[0] for k, _ in kpts] if self.comm.size > 1 else None
        self.owner = kpar.deal_kpoints(self.nk, self.comm.size, costs)
        self.kglobal = [k for k in range(self.nk) if self.owner[k] == self.comm.rank]
        tm = self.setup_times = {}
        t = time.perf_counter()
        # radial projector tables per species (nonlocal_context.zig builds them once per species);
        # run_scf_many shares them across its cells through table_cache
        tc = table_cache if table_cache is not None else {}
        tables = []
        resident = bool(getattr(backend, "resident", False))
        for sp in c.species:
            key = (sp.name, p.ecut)
            if key not in tc:
                if resident:  # one kernel launch per beta (dftcuda_radial_table)
                    gmax = 1.5 * math.sqrt(2.0 * p.ecut)
                    tc[key] = [backend.dz.radial_table(l, sp.r, beta, sp.rab, gmax) for (l, beta) in sp.betas]
                else:
                    tc[key] = [sysm.radial_table(sp, i, p.ecut) for i in range(len(sp.betas))]
            tables.append(tc[key])
        tm["radial_tables"], t = time.perf_counter() - t, time.perf_counter()
        # resident backends: density, potential and mixing history on the device (csrc/potential.cu),
        # the ionic local potential built there too
        self.dev = bool(getattr(backend, "resident", False))
        if self.dev:
            import torch

            self.pot = backend.dz.PotentialContext(dims, self.vol, c.recip, history=max(1, p.pulay_history), functional=p.xc)
            _, self.vloc_d = self.pot.ionic_radial([sp.mesh for sp in c.species], c.atom_species, c.positions, 4.0 * p.ecut,
                                                   device=True)
            self.vloc_r = self.vloc_d.cpu().numpy()
        else:
            if p.xc != "lda":
                raise ValueError("ScfParams.xc = 'pbe' needs the resident driver (GpuBackend(resident=True))")
            self.vloc_r = sysm.local_potential(c, dims, p.ecut)
        tm["local_potential"], t = time.perf_counter() - t, time.perf_counter()
        if self.dev:  # basis and projector rows on the device too (dftcuda_plane_wave_basis, dftcuda_projector_phi)
            self.kin = [sysm.kpoint_inputs_device(backend.dz, c, p.ecut, kpts[k][0], dims=dims, local_r=self.vloc_r, tables=tables)
                        for k in self.kglobal]
        else:
            self.kin = [sysm.kpoint_inputs(c, p.ecut, kpts[k][0], dims=dims, local_r=self.vloc_r, tables=tables) for k in self.kglobal]
        self.kweights = [w for _, w in kpts]
        tm["kpoint_inputs"], t = time.perf_counter() - t, time.perf_counter()
        backend.setup(self.kin)
        tm["contexts"], t = time.perf_counter() - t, time.perf_counter()
        if not self.dev:  # the host potential path's G-vector table
            self.g2 = g_vectors(dims, c.recip)
            self.gmask = self.g2 > 1e-12
        self.dielec = None
        if p.diemac > 1.0:
            g2 = self.g2 if not self.dev else g_vectors(dims, c.recip)
            x = p.dielng * p.dielng * g2
            self.dielec = np.where(g2 < 1e-12, 1.0 / p.diemac, (x + 1.0 / p.diemac) / (x + 1.0))
        self.nelec = c.nelec
        self.nocc = int(math.ceil(self.nelec / 2.0 - 1e-12))
        self.nbands = max(p.nbands, self.nocc)
        if p.initial_density is None:
            self.rho = np.full(N, self.nelec / self.vol)  # init_rho_from_user_or_flat (run_state.zig:98-115)
        else:
            self.rho = np.asarray(p.initial_density, dtype=np.float64).copy()
            if self.rho.size != N:
                raise ValueError("initial_density size does not match the FFT grid")
        if self.dev:
            import torch

            self.rho = torch.from_numpy(self.rho).cuda()
            self.v_hxc, _ = self.pot.hxc(self.rho)
        else:
            self.v_hxc = self.hxc_g(self.rho)
        self.mixer = PulayMixer(p.pulay_history)
        self.vectors = [None] * len(self.kin)  # this rank's k-points, in kglobal order
        t = time.perf_counter()
        self.e_ion = ewald_energy(c.cell, np.array([c.species[s].z_val for s in c.atom_species]), c.positions)
        tm["ewald"] = time.perf_counter() - t
        # psp_core = sum of epsatm over the atoms x N_e / Omega (energy.zig:350-365)
        eps = [sysm.epsatm(sp) for sp in c.species]
        self.psp_core = sum(eps[s] for s in c.atom_species) * self.nelec / self.vol
        self.history = []
        self.energy = float("nan")
        self.terms = {}
        self.converged = False
        self.done = False
        self.values = []
        self.it = 0

    def to_g(self, fr):
        d = self.dims
        return np.fft.fftn(fr.reshape(d[2], d[1], d[0])).ravel() / self.N

    def to_r(self, fg):
        d = self.dims
        return np.fft.ifftn(fg.reshape(d[2], d[1], d[0])).ravel().real * self.N

    def hxc_g(self, rho):
        rg = self.to_g(rho)
        vh = np.zeros_like(rg)
        vh[self.gmask] = 8.0 * math.pi * rg[self.gmask] / self.g2[self.gmask]
        _, vxc = lda_pz(rho)
        return vh + self.to_g(vxc)

    def begin(self):
        """Start the next iteration: set V(r); returns the eigensolver options and warm starts."""
        p = self.p
        self.it += 1
        local_r = self.pot.real(self.v_hxc, self.vloc_d) if self.dev else self.vloc_r + self.to_r(self.v_hxc)
        self.backend.set_vloc(local_r)
        warm = self.it <= p.warmup_steps
        opts = dict(max_iter=p.warmup_max_iter if warm else p.iterative_max_iter, tol=p.warmup_tol if warm else p.iterative_tol)
        inits = [self.vectors[k] if (p.reuse_vectors and self.vectors[k] is not None) else None for k in range(len(self.kin))]
        return opts, inits

    def finish(self, results):
        """Occupations, density, energy, convergence test and mixing from the eigenpairs of begin()
        (``results`` for this rank's k-points).  With several ranks the eigenvalue table and the
        density are sum-reduced over them; everything after that is replicated."""
        p, c, N, vol = self.p, self.c, self.N, self.vol
        nbands, nelec = self.nbands, self.nelec
        table = np.zeros((self.nk, nbands))
        for i, (ev, vec) in enumerate(results):
            table[self.kglobal[i]] = np.asarray(ev)[:nbands]
            self.vectors[i] = vec
        if self.comm.size > 1:
            table = self.comm.sum(table)
        self.values = values = [table[k] for k in range(self.nk)]
        dev_occ = None
        if p.smearing and self.dev:
            # Fermi level, occupations and the band / entropy sums in FP64 on the device
            mu, occ_tab, eb, es = self.backend.dz.fermi_occupations(table, self.kweights, nelec, p.smearing)
            occs = [occ_tab[k] for k in range(self.nk)]
            dev_occ = (eb, es)
        elif p.smearing:
            mu = fermi_level(nelec, p.smearing, self.kweights, values)
            occs = [fd_occ(v, mu, p.smearing) for v in values]
        else:
            occ = np.zeros(nbands)
            occ[: self.nocc - 1] = 1.0
            occ[self.nocc - 1] = nelec / 2.0 - (self.nocc - 1)
            occs = [occ for _ in values]
        self.occs = occs
        if self.dev:
            import torch

            rho_out = torch.zeros(N, dtype=torch.float64, device="cuda")
        else:
            rho_out = np.zeros(N)
        e_band = 0.0
        e_ent = 0.0
        if dev_occ is not None:
            e_band, e_ent = dev_occ[0], p.smearing * dev_occ[1]
        else:
            for k in range(self.nk):
                wts = self.kweights[k] * occs[k] * 2.0
                e_band += float(np.dot(wts, values[k]))
                if p.smearing:
                    e_ent += self.kweights[k] * 2.0 * p.smearing * float(entropy_term(occs[k]).sum())
        for i, k in enumerate(self.kglobal):
            self.backend.density(i, self.vectors[i], self.kweights[k] * occs[k] * 2.0, rho_out)
        if self.comm.size > 1:
            rho_out = self.comm.sum(rho_out)
        if self.dev:
            diff = math.sqrt(float(((rho_out - self.rho) ** 2).mean()))
        else:
            diff = math.sqrt(float(np.mean((rho_out - self.rho) ** 2)))
        if hasattr(self.backend, "observe"):
            self.backend.observe(diff)
        # energy of rho_out with eigenvalues from V_in (energy.zig:372-396)
        if self.dev:
            v_out_d, terms = self.pot.hxc(rho_out, v_in=self.v_hxc)
            e_h, e_xc, int_vin_rho = terms["e_hartree"], terms["e_xc"], terms["int_vin_rho"]
        else:
            rg = self.to_g(rho_out)
            gm = self.gmask
            e_h = 0.5 * vol * float(np.sum(8.0 * math.pi * np.abs(rg[gm]) ** 2 / self.g2[gm]))
            fxc, _ = lda_pz(rho_out)
            dv = vol / N
            e_xc = float(fxc.sum()) * dv
            v_in_r = self.to_r(self.v_hxc)
            int_vin_rho = float(np.dot(v_in_r, rho_out)) * dv
        self.energy = e_band - int_vin_rho + e_h + e_xc + self.e_ion + self.psp_core - e_ent
        self.terms = dict(band=e_band, hartree=e_h, xc=e_xc, vin_rho=int_vin_rho, ion_ion=self.e_ion, psp_core=self.psp_core, entropy=e_ent)
        self.history.append((self.it, self.energy, diff, time.perf_counter() - self.t0))
        if self.verbose and self.comm.rank == 0:
            print(f"scf {self.it:3d}  E={self.energy:.10f} Ry  drho={diff:.3e}", flush=True)
        if p.energy_target is not None and p.energy_tol_per_atom is not None:
            if abs(self.energy - p.energy_target) / len(c.atom_species) < p.energy_tol_per_atom:
                self.converged = self.done = True
                self.rho = rho_out
                return True
        if diff < p.convergence:
            self.converged = self.done = True
            self.rho = rho_out
            return True
        # Pulay from the reference's 0-based iteration index pulay_start on (scf.zig:164, 495: the
        # loop counter starts at 0); self.it counts from 1
        pulay = self.it - 1 >= p.pulay_start
        if self.dev:
            import torch

            resid = v_out_d - self.v_hxc
            if pulay:
                if self.dielec is not None:
                    if not torch.is_tensor(self.dielec):
                        self.dielec = torch.from_numpy(self.dielec).to(resid.device)
                    resid = resid * self.dielec
                x = torch.view_as_real(self.v_hxc).reshape(-1).clone()
                self.pot.pulay_mix(x, torch.view_as_real(resid).reshape(-1).contiguous(), p.mixing_beta)
                self.v_hxc = torch.view_as_complex(x.view(-1, 2))
            else:
                self.v_hxc = self.v_hxc + p.mixing_beta * resid
        else:
            resid = self.hxc_g(rho_out) - self.v_hxc
            if pulay:
                if self.dielec is not None:
                    resid = resid * self.dielec
                flat = self.mixer.mix(np.concatenate([self.v_hxc.real, self.v_hxc.imag]), np.concatenate([resid.real, resid.imag]), p.mixing_beta)
                self.v_hxc = flat[:N] + 1j * flat[N:]
            else:
                self.v_hxc = self.v_hxc + p.mixing_beta * resid
        self.rho = rho_out
        if self.it >= p.max_iter:
            self.done = True
        return self.done

    def result(self) -> ScfResult:
        natom = len(self.c.atom_species)
        rho = self.rho.cpu().numpy() if self.dev else self.rho
        return ScfResult(self.converged, self.it, self.energy, self.energy / natom, self.values, self.terms, rho, self.history,
                         time.perf_counter() - self.t0)

    def forces(self) -> np.ndarray:
        """Hellmann-Feynman forces (natoms, 3, Ry/bohr) of the last iteration's density and bands
        (compute_forces, forces/forces.zig:785-851, without NLCC, PAW or dispersion terms): local
        pseudopotential (device), nonlocal (device, summed over this rank's k-points and over the
        ranks) and ion-ion (host Ewald)."""
        if not self.dev:
            raise ValueError("forces need the resident driver (GpuBackend(resident=True))")
        c, p = self.c, self.p
        natoms = len(c.atom_species)
        f_loc = self.pot.local_forces_radial([sp.mesh for sp in c.species], c.atom_species, c.positions, self.rho, 4.0 * p.ecut)
        f_nl = np.zeros((natoms, 3))
        for i, k in enumerate(self.kglobal):
            w = self.kweights[k] * np.asarray(self.occs[k]) * 2.0
            f_nl += self.backend.nonlocal_forces(i, self.vectors[i], w, natoms)
        if self.comm.size > 1:
            f_nl = self.comm.sum(f_nl)
        f_ion = ewald_forces(c.cell, np.array([c.species[s].z_val for s in c.atom_species]), c.positions)
        self.force_terms = {"local": f_loc, "nonlocal": f_nl, "ion_ion": f_ion}
        return f_loc + f_nl + f_ion

    def close(self):
        if self.dev:
            self.pot.close()


def run_scf(c: sysm.Crystal, p: ScfParams, backend, verbose: bool = False, comm=None, forces: bool = False) -> ScfResult:
    """The SCF loop.  ``comm`` (a kpar.KpointComm) deals the k-points over the ranks of a process
    group; every rank returns the same result.  forces: also the Hellmann-Feynman forces of the
    final state (resident driver)."""
    st = ScfState(c, p, backend, verbose, comm)
    try:
        r = _run(st, backend)
        if forces:
            r.forces = st.forces()
        return r
    finally:
        st.close()


def _run(st, backend) -> ScfResult:
    while not st.done:
        opts, inits = st.begin()
        diags = [inp.basis.kinetic for inp in st.kin]
        if hasattr(backend, "eig_all"):
            # every k-point's solve at once (the k-point worker loop, kpoint/workers.zig:133-180)
            res = backend.eig_all(diags, st.nbands, opts, inits)
        else:
            res = [backend.eig(k, diags[k], st.nbands, opts, inits[k]) for k in range(len(st.kin))]
        st.finish(res)
    return st.result()


def run_scf_many(dz, cells, p: ScfParams, precision: str = "fp64", initial_densities=None, resident: bool = False):
    """Independent SCF runs of many cells advanced together: each iteration, the eigensolves of
    every (cell, k-point) pair still running go through one lockstep batch
    (dftcuda_eig_solve_batch) on their contexts' streams.  All cells need the same band count.
    resident: every cell's eigenvectors, density, potential and mixing stay on the device."""
    t0 = time.perf_counter()
    phases = {"setup": 0.0, "begin": 0.0, "eig": 0.0, "finish": 0.0}
    states = []
    tables = {}  # radial tables shared by the cells' species
    for i, c in enumerate(cells):
        pi = p if initial_densities is None else ScfParams(**{**p.__dict__, "initial_density": initial_densities[i]})
        states.append(ScfState(c, pi, GpuBackend(dz, precision, resident=resident), table_cache=tables))
    phases["setup"] = time.perf_counter() - t0
    if len({st.nbands for st in states}) != 1:
        raise ValueError("run_scf_many: the cells need the same number of bands")
    nb = states[0].nbands
    while True:
        active = [st for st in states if not st.done]
        if not active:
            break
        groups = {}
        begun = []
        tb = time.perf_counter()
        for st in active:
            opts, inits = st.begin()
            begun.append((st, inits))
            groups.setdefault((opts["max_iter"], opts["tol"]), []).append((st, inits))
        te = time.perf_counter()
        phases["begin"] += te - tb
        out = {}
        for (mi, tol), members in groups.items():
            ctxs, diags, inits = [], [], []
            for st, iv in members:
                ctxs += st.backend._active()
                diags += [inp.basis.kinetic for inp in st.kin]
                inits += iv
            rs = dz.hermitian_eigen_decomp_iterative_batch(ctxs, diags, nb, dz.Options(max_iter=mi, tol=tol), inits,
                                                            device=resident)
            o = 0
            for st, _ in members:
                nk = len(st.kin)
                out[id(st)] = [(r.values, r.vectors) for r in rs[o:o + nk]]
                o += nk
        tf = time.perf_counter()
        phases["eig"] += tf - te
        for st, _ in begun:
            st.finish(out[id(st)])
        phases["finish"] += time.perf_counter() - tf
    results = [st.result() for st in states]
    for st in states:
        st.close()
        st.backend.close()
    setup = {}
    for st in states:
        for k, v in st.setup_times.items():
            setup[k] = setup.get(k, 0.0) + v
    phases.update({f"setup_{k}": v for k, v in setup.items()})
    run_scf_many.last_phases = {k: round(v, 3) for k, v in phases.items()}
    return results, time.perf_counter() - t0
