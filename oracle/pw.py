"""Plane-wave basis, FFT grid and G-sphere <-> FFT-box maps (oracle; test infrastructure only).

Restates:
  src/features/math/math.zig:131-142          reciprocal()
  src/features/plane_wave/basis.zig:26-74     generate()
  src/features/scf/pw_grid.zig:54-72          auto_grid(), min_index()
  src/lib/fft/sizing.zig:1-15                 next_fft_size()
  src/features/scf/pw_grid_map.zig:18-117     PwGridMap (indices, fft_indices, scatter/gather)
  src/features/scf/fft_grid.zig:407-438       build_fft_index_map(), index_to_freq()
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903


def reciprocal(cell: np.ndarray) -> np.ndarray:
    """Rows b_i = 2*pi*(a_j x a_k)/Omega (math.zig:131-142)."""
    a1, a2, a3 = cell
    vol = float(np.dot(a1, np.cross(a2, a3)))
    s = 2.0 * math.pi / vol
    return np.array([np.cross(a2, a3) * s, np.cross(a3, a1) * s, np.cross(a1, a2) * s])


def cell_volume(cell: np.ndarray) -> float:
    return abs(float(np.dot(cell[0], np.cross(cell[1], cell[2]))))


@dataclass
class Basis:
    """G-sphere for one k (basis.zig:5-12): Miller indices, G, k+G and |k+G|^2 (Ry)."""

    hkl: np.ndarray  # int32 [n,3]
    cart: np.ndarray  # [n,3]
    kpg: np.ndarray  # [n,3]
    kinetic: np.ndarray  # [n]

    @property
    def n(self) -> int:
        return int(self.hkl.shape[0])


def generate_basis(recip: np.ndarray, ecut_ry: float, k_cart) -> Basis:
    """basis.zig:26-74: loop h (outer), k, l (inner) over [-max_n, max_n], keep |k+G|^2 <= ecut."""
    k_cart = np.asarray(k_cart, dtype=np.float64)
    min_b = min(np.linalg.norm(recip[0]), np.linalg.norm(recip[1]), np.linalg.norm(recip[2]))
    gmax = math.sqrt(ecut_ry)
    max_n = int(math.ceil(gmax / min_b)) + 1
    r = np.arange(-max_n, max_n + 1, dtype=np.int32)
    h, k, l = np.meshgrid(r, r, r, indexing="ij")  # h outermost, l innermost in C order
    hkl = np.stack([h.ravel(), k.ravel(), l.ravel()], axis=1)
    # Same summation order as the reference: (b1*h + b2*k) + b3*l, then k + G.
    g = (recip[0][None, :] * hkl[:, 0:1] + recip[1][None, :] * hkl[:, 1:2]) + recip[2][None, :] * hkl[:, 2:3]
    kpg = k_cart[None, :] + g
    kin = kpg[:, 0] * kpg[:, 0] + kpg[:, 1] * kpg[:, 1] + kpg[:, 2] * kpg[:, 2]
    keep = kin <= ecut_ry
    return Basis(hkl=hkl[keep].astype(np.int32), cart=g[keep], kpg=kpg[keep], kinetic=kin[keep])


def is_fft_size(n: int) -> bool:
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def next_fft_size(value: int) -> int:
    """sizing.zig:1-15: next 2,3,5-smooth integer >= value."""
    if value <= 1:
        return 1
    n = value
    while not is_fft_size(n):
        n += 1
    return n


def auto_grid(ecut_ry: float, recip: np.ndarray, grid_scale: float = 1.0):
    """pw_grid.zig:54-68: n_i = next_fft_size(max(2*ceil(max(2,scale)*sqrt(ecut)/|b_i|)+1, 3))."""
    scale = grid_scale if grid_scale > 0.0 else 1.0
    gmax = max(2.0, scale) * math.sqrt(ecut_ry)
    out = []
    for i in range(3):
        b = float(np.linalg.norm(recip[i]))
        n = int(math.ceil(gmax / b)) * 2 + 1
        out.append(next_fft_size(max(n, 3)))
    return tuple(out)


def min_index(n: int) -> int:
    """pw_grid.zig:70-72."""
    return -(n // 2)


def index_to_freq(i: int, n: int) -> int:
    """fft_grid.zig:434-438."""
    half = (n - 1) // 2
    return i if i <= half else i - n


@dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    volume: float

    @property
    def min_h(self):
        return min_index(self.nx)

    @property
    def min_k(self):
        return min_index(self.ny)

    @property
    def min_l(self):
        return min_index(self.nz)

    @property
    def count(self):
        return self.nx * self.ny * self.nz


def build_fft_index_map(grid: Grid) -> np.ndarray:
    """fft_grid.zig:407-431: FFT-order position -> centred-grid position."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    fx = np.array([index_to_freq(i, nx) for i in range(nx)]) - grid.min_h
    fy = np.array([index_to_freq(i, ny) for i in range(ny)]) - grid.min_k
    fz = np.array([index_to_freq(i, nz) for i in range(nz)]) - grid.min_l
    zz, yy, xx = np.meshgrid(fz, fy, fx, indexing="ij")
    return (xx + nx * (yy + ny * zz)).ravel().astype(np.int64)


class PwGridMap:
    """pw_grid_map.zig:8-117."""

    def __init__(self, basis: Basis, grid: Grid):
        hi = basis.hkl[:, 0] - grid.min_h
        ki = basis.hkl[:, 1] - grid.min_k
        li = basis.hkl[:, 2] - grid.min_l
        if (hi < 0).any() or (ki < 0).any() or (li < 0).any():
            raise ValueError("InvalidGrid")
        if (hi >= grid.nx).any() or (ki >= grid.ny).any() or (li >= grid.nz).any():
            raise ValueError("InvalidGrid")
        self.grid = grid
        self.indices = (hi + grid.nx * (ki + grid.ny * li)).astype(np.int64)
        self.fft_indices = None

    def build_fft_indices(self, fft_index_map: np.ndarray):
        """pw_grid_map.zig:58-78: invert the FFT index map, then PW -> FFT-order position."""
        inv = np.empty_like(fft_index_map)
        inv[fft_index_map] = np.arange(fft_index_map.size)
        self.fft_indices = inv[self.indices]
        return self.fft_indices

    def scatter(self, coeffs, out):
        out[:] = 0
        out[self.indices] = coeffs

    def gather(self, data):
        return data[self.indices].copy()

    def scatter_fft(self, coeffs, out, scale):
        """pw_grid_map.zig:94-104."""
        out[:] = 0
        out[self.fft_indices] = coeffs * scale

    def gather_fft(self, data, scale):
        """pw_grid_map.zig:107-116."""
        return data[self.fft_indices] * scale


def fft_indices_direct(hkl: np.ndarray, grid: Grid) -> np.ndarray:
    """Same result as PwGridMap.build_fft_indices: position (h mod nx) + nx*((k mod ny) + ny*(l mod nz))."""
    x = np.mod(hkl[:, 0], grid.nx)
    y = np.mod(hkl[:, 1], grid.ny)
    z = np.mod(hkl[:, 2], grid.nz)
    return (x + grid.nx * (y + grid.ny * z)).astype(np.int64)
