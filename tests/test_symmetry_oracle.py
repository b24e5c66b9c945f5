"""The density-symmetrisation oracle (oracle/symmetry.py) on the CPU: the space-group search on
diamond cells, and the properties the symmetrised density must have (every operation leaves it
unchanged, a second pass changes nothing, the charge is kept, a density that already has the
crystal's symmetry comes back as it was)."""
import importlib
import math

import numpy as np

import dftzig_loader
from oracle import potential as op
from oracle import symmetry as sy

dftzig_loader.load()
system = importlib.import_module("dftzig_b200.system")


def _ops(name):
    c = system.crystal(name)
    cell = np.asarray(c.cell, dtype=np.float64)
    frac = np.asarray(c.positions, dtype=np.float64) @ np.linalg.inv(cell)
    return c, cell, frac, sy.symmetry_ops(cell, frac, c.atom_species)


def _band_limited(dims, recip, gmax2, seed):
    """A random real density with Fourier components only inside |G|^2 < gmax2 (well inside the box,
    so that rotated G vectors never wrap)."""
    rng = np.random.default_rng(seed)
    n = dims[0] * dims[1] * dims[2]
    g2 = op.g2_table(dims, recip)
    rg = op.to_g(rng.normal(size=n), dims)
    return 0.05 + 0.01 * op.to_r(np.where(g2 < gmax2, rg, 0.0), dims)


def test_space_group_orders_of_diamond_cells():
    assert len(_ops("si2")[3]) == 48  # O_h, primitive cell
    assert len(_ops("si8")[3]) == 192  # O_h x 4 face-centring translations, conventional cell
    # the identity with zero translation is one of them, and k_rot = (rot^-1)^T
    for rot, k_rot, _ in _ops("si2")[3]:
        assert np.array_equal(k_rot @ rot.T, np.eye(3, dtype=np.int64))


def test_symmetrised_density_is_invariant_and_idempotent():
    c, cell, frac, ops = _ops("si2")
    dims = (16, 16, 16)
    recip = 2 * math.pi * np.linalg.inv(cell).T
    rho = _band_limited(dims, recip, 6.0, 1)
    sym = sy.symmetrize_density(rho, dims, ops)
    assert abs(sym.mean() - rho.mean()) < 1e-14  # G = 0 kept: the charge is unchanged
    assert np.abs(sy.symmetrize_density(sym, dims, ops) - sym).max() < 1e-13
    # every operation maps the symmetrised density onto itself: in G space,
    # rho(k_rot G) e^{-2 pi i G.t} = rho(G)
    nx, ny, nz = dims
    rg = op.to_g(sym, dims).reshape(nz, ny, nx)
    f = [np.where(np.arange(n) <= (n - 1) // 2, np.arange(n), np.arange(n) - n) for n in dims]
    h, k, l = f[0][None, None, :], f[1][None, :, None], f[2][:, None, None]
    for _, kr, t in ops:
        hh = kr[0, 0] * h + kr[0, 1] * k + kr[0, 2] * l
        kk = kr[1, 0] * h + kr[1, 1] * k + kr[1, 2] * l
        ll = kr[2, 0] * h + kr[2, 1] * k + kr[2, 2] * l
        moved = rg[np.mod(ll, nz), np.mod(kk, ny), np.mod(hh, nx)] * np.exp(-2j * math.pi * (h * t[0] + k * t[1] + l * t[2]))
        assert np.abs(moved - rg).max() < 1e-14
    # a random density is not symmetric: the pass does change it
    assert np.abs(sym - rho).max() > 1e-4


def test_symmetric_density_is_unchanged():
    """Gaussians on the atoms of the conventional Si8 cell (with its 192 operations) already have
    the crystal's symmetry."""
    c, cell, frac, ops = _ops("si8")
    dims = (24, 24, 24)
    n = dims[0] * dims[1] * dims[2]
    grid = np.stack(np.meshgrid(*[np.arange(d) / d for d in dims], indexing="ij"), axis=-1)  # x, y, z
    grid = grid.transpose(2, 1, 0, 3).reshape(n, 3)  # x fastest
    rho = np.zeros(n)
    for f in frac:
        d = grid - f
        d -= np.rint(d)
        r2 = ((d @ cell) ** 2).sum(axis=1)
        rho += np.exp(-r2 / 0.8)
    sym = sy.symmetrize_density(rho, dims, ops)
    assert np.abs(sym - rho).max() < 1e-10 * np.abs(rho).max()


def _si_conventional(swap):
    """The cells of the reference's space-group tests (src/tests.zig:46-135): diamond Si, a = 5.431,
    eight atoms; `swap` exchanges the first two lattice vectors (a left-handed basis)."""
    a = 5.431
    h, q, t = a / 2, a / 4, 3 * a / 4
    cell = np.array([[0.0, a, 0.0], [a, 0.0, 0.0], [0.0, 0.0, a]]) if swap else np.eye(3) * a
    pos = np.array([[0, 0, 0], [0, h, h], [h, 0, h], [h, h, 0], [q, q, q], [q, t, t], [t, q, t], [t, t, q]], dtype=np.float64)
    return cell, pos @ np.linalg.inv(cell)


def test_reference_space_group_cells():
    """Fd-3m (No. 227, the reference's expected group) in the conventional cell: 48 rotations x 4
    face-centring translations, in both bases; symmetrising atom-centred Gaussians in the swapped
    basis returns them unchanged."""
    for swap in (False, True):
        cell, frac = _si_conventional(swap)
        ops = sy.symmetry_ops(cell, frac, [0] * 8)
        assert len(ops) == 192
        assert sum(1 for rot, _, t in ops if np.array_equal(rot, np.eye(3, dtype=np.int64))) == 4  # pure translations
    cell, frac = _si_conventional(True)
    ops = sy.symmetry_ops(cell, frac, [0] * 8)
    dims = (20, 20, 20)
    n = dims[0] * dims[1] * dims[2]
    grid = np.stack(np.meshgrid(*[np.arange(d) / d for d in dims], indexing="ij"), axis=-1).transpose(2, 1, 0, 3).reshape(n, 3)
    rho = np.zeros(n)
    for f in frac:
        d = grid - f
        d -= np.rint(d)
        rho += np.exp(-((d @ cell) ** 2).sum(axis=1) / 0.6)
    assert np.abs(sy.symmetrize_density(rho, dims, ops) - rho).max() < 1e-10 * rho.max()


def test_identity_only_is_a_copy():
    dims = (6, 5, 4)
    rho = np.random.default_rng(3).random(6 * 5 * 4)
    ident = [(np.eye(3, dtype=np.int64), np.eye(3, dtype=np.int64), np.zeros(3))]
    assert np.array_equal(sy.symmetrize_density(rho, dims, ident), rho)
