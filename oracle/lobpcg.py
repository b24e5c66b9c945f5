"""dft-zig's serial block-Davidson ("LOBPCG") eigensolver (oracle; test infrastructure only).

Restates src/features/linalg/lobpcg/serial.zig:55-307 and the helpers in
src/features/linalg/lobpcg/common.zig:
  44-52    Options
  113-143  combine_columns_matrix  (V.C zgemm)
  214-226  precondition            (r_i/(diag_i - lambda), |den| >= 1e-8 keeping the sign)
  231-259  build_projected         (T = V^H W, then (T+T^H)/2 with a real diagonal)
  263-284  orthonormalize_vector   (modified Gram-Schmidt, then dznrm2 normalisation)
  287-312  init_random_vectors / orthonormalize_all (3 random retries)
  314-319  next_rand01             (LCG s = s*6364136223846793005 + 1, (s>>11)/2^53)
  440-508  hermitian_eigen_decomp_small (LAPACK zheev; numpy.linalg.eigh here)
Only the standard problem (apply_s = null) is restated: the norm-conserving
path never sets apply_s (kpoint/solve.zig:309-315).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

MASK64 = (1 << 64) - 1


@dataclass
class Options:
    max_iter: int = 40
    tol: float = 1e-6
    max_subspace: int = 0
    block_size: int = 0
    init_diagonal: bool = False
    init_vectors: Optional[np.ndarray] = None  # (cols, n)
    init_vectors_cols: int = 0


@dataclass
class Operator:
    n: int
    apply_batch: Callable  # (X (m,n)) -> (m,n)


class Lcg:
    def __init__(self, seed=0x6F3D3CBE):
        self.s = seed

    def next01(self) -> float:
        self.s = (self.s * 6364136223846793005 + 1) & MASK64
        return float(self.s >> 11) / 9007199254740992.0


def lcg_stream(s0: int, count: int):
    """The next ``count`` LCG states after s0, computed in closed form
    s_k = a^k s0 + sum_{j<k} a^j (mod 2^64) with numpy's wrapping uint64 arithmetic.
    Returns (states, last_state)."""
    a = np.uint64(6364136223846793005)
    powers = np.empty(count + 1, dtype=np.uint64)
    powers[0] = 1
    powers[1:] = a
    with np.errstate(over="ignore"):
        powers = np.cumprod(powers, dtype=np.uint64)  # a^0 .. a^count
        geo = np.cumsum(powers, dtype=np.uint64)  # sum_{j<=k} a^j
        states = powers[1:] * np.uint64(s0) + geo[:-1]
    return states, int(states[-1]) if count else s0


def random_block(n: int, m: int, rng: Lcg) -> np.ndarray:
    """init_random_vectors (common.zig:287-295): column by column, (re, im) pairs."""
    if n * m == 0:
        return np.zeros((m, n), dtype=np.complex128)
    states, rng.s = lcg_stream(rng.s, 2 * n * m)
    vals = (states >> np.uint64(11)).astype(np.float64) / 9007199254740992.0 - 0.5
    return (vals[0::2] + 1j * vals[1::2]).reshape(m, n)


def random_vector(n: int, rng: Lcg) -> np.ndarray:
    return random_block(n, 1, rng)[0]


def orthonormalize_vector(v: np.ndarray, basis: np.ndarray, m: int) -> float:
    """common.zig:263-284 (MGS against basis[0:m]); v updated in place, returns the pre-scale norm."""
    for j in range(m):
        dot = np.vdot(basis[j], v)
        v -= dot * basis[j]
    norm = float(np.linalg.norm(v))
    if norm > 0.0:
        v *= 1.0 / norm
    return norm


def orthonormalize_all(v: np.ndarray, m: int, rng: Lcg):
    """common.zig:298-312."""
    n = v.shape[1]
    for col in range(m):
        for _ in range(3):
            norm = orthonormalize_vector(v[col], v, col)
            if norm > 1e-8:
                break
            v[col] = random_vector(n, rng)
        if np.linalg.norm(v[col]) < 1e-8:
            raise ValueError("InvalidMatrixSize")


def precondition(diag: np.ndarray, lam: float, r: np.ndarray) -> np.ndarray:
    den = diag - lam
    small = np.abs(den) < 1e-8
    den = np.where(small, np.where(den >= 0.0, 1e-8, -1e-8), den)
    return r * (1.0 / den)


def build_projected(v: np.ndarray, w: np.ndarray, m: int) -> np.ndarray:
    t = v[:m].conj() @ w[:m].T  # T[i,j] = <v_i|w_j>
    t = 0.5 * (t + t.conj().T)
    t[np.diag_indices(m)] = t.diagonal().real
    return t


@dataclass
class EigenResult:
    values: np.ndarray
    vectors: np.ndarray  # (nbands, n)
    iterations: int
    converged: bool
    h_applies: int


def solve(op: Operator, diag: np.ndarray, nbands: int, opts: Options) -> EigenResult:
    """serial.zig:55-307."""
    n = op.n
    if nbands == 0 or n == 0:
        return EigenResult(np.zeros(0), np.zeros((0, n), complex), 0, True, 0)
    max_sub = min(n, 4 * nbands + 8) if opts.max_subspace == 0 else min(n, max(opts.max_subspace, nbands))
    block = min(max_sub, nbands + 4) if opts.block_size == 0 else min(max_sub, max(opts.block_size, nbands))
    v = np.zeros((max_sub, n), dtype=np.complex128)
    w = np.zeros((max_sub, n), dtype=np.complex128)
    rng = Lcg()
    m = block
    init_cols = 0
    if opts.init_vectors is not None:
        cols = nbands if opts.init_vectors_cols == 0 else opts.init_vectors_cols
        init_cols = min(m, cols)
    if opts.init_diagonal:
        order = np.argsort(diag, kind="stable")
        for col in range(m):
            v[col, order[col]] = 1.0
    else:
        v[:m] = random_block(n, m, rng)
    if opts.init_vectors is not None:
        v[:init_cols] = np.asarray(opts.init_vectors).reshape(-1, n)[:init_cols]
    orthonormalize_all(v, m, rng)
    w[:m] = op.apply_batch(v[:m])
    applies = m
    last_values = np.zeros(nbands)
    ritz = None
    for it in range(opts.max_iter):
        t = build_projected(v, w, m)
        evals, evecs = np.linalg.eigh(t)
        last_values = evals[:nbands].copy()
        c = evecs[:, :nbands]
        ritz = (v[:m].T @ c).T  # (nbands, n)
        res = (w[:m].T @ c).T
        norms = np.empty(nbands)
        for b in range(nbands):
            res[b] -= evals[b] * ritz[b]
            norms[b] = np.linalg.norm(res[b])
        if norms.max() < opts.tol:
            return EigenResult(last_values, ritz, it + 1, True, applies)
        added = 0
        for b in range(nbands):
            if m + added >= max_sub:
                break
            if norms[b] < opts.tol:
                continue
            q = precondition(diag, evals[b], res[b])
            v[m + added] = q
            norm = orthonormalize_vector(v[m + added], v, m + added)
            if norm < 1e-8:
                continue
            added += 1
        if added > 0:
            w[m : m + added] = op.apply_batch(v[m : m + added])
            applies += added
        if added == 0:
            return EigenResult(last_values, ritz, it + 1, True, applies)
        if m + added >= max_sub:
            v[:nbands] = ritz
            m = nbands
            orthonormalize_all(v, m, rng)
            w[:m] = op.apply_batch(v[:m])
            applies += m
            continue
        m += added
    return EigenResult(last_values, ritz, opts.max_iter, False, applies)
