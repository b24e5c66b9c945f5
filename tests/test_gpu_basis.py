"""Plane-wave basis and projector tables built on the device, against the oracle.

* dftcuda_plane_wave_basis vs the oracle's plane_wave.generate (basis.zig:26-74): the same Miller
  triples in the same order, and G, k+G and |k+G|^2 equal bit for bit, at the configs' cells and
  cutoffs (Si2 20 Ry off-Gamma, Al4 25 Ry, SiGe8 20 Ry, Si216 25 Ry at Gamma: 61,565 plane waves).
* dftcuda_projector_phi vs the oracle's fill_nonlocal_phi (4 pi R(|q|) Y_lm(q), RadialTable.eval,
  real Y_lm for l = 0..4) to 1e-13 of the largest entry, including q = 0 and q beyond the table.
"""
import math

import numpy as np
import pytest

from oracle import pseudo, pw
from tests.helpers import cell

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,seed,ecut,kfrac", [("si2", 1, 20.0, (0.25, 0.125, 0.0)), ("al4", 2, 25.0, (0.1, 0.2, 0.3)),
                                                  ("sige8", 1, 20.0, (0.25, 0.25, 0.25)), ("si216", 3, 25.0, (0.0, 0.0, 0.0))])
def test_basis_matches_oracle_bit_for_bit(dz, name, seed, ecut, kfrac):
    c = cell(name, seed)
    k = np.asarray(kfrac, float) @ c.recip
    hkl, g, q, kin = dz.plane_wave_basis(c.recip, ecut, k)
    ref = pw.generate_basis(c.recip, ecut, k)
    assert hkl.shape == ref.hkl.shape
    assert np.array_equal(hkl, ref.hkl)
    assert np.array_equal(g, ref.cart) and np.array_equal(q, ref.kpg) and np.array_equal(kin, ref.kinetic)
    if name == "si216":
        assert len(kin) == 61565


def test_basis_size_query_and_capacity(dz):
    import ctypes as ct

    c = cell("si2", 1)
    lib = dz.load_library()
    recip = np.ascontiguousarray(c.recip.reshape(9))
    k = np.zeros(3)
    n = ct.c_size_t(0)
    assert lib.dftcuda_plane_wave_basis(recip.ctypes.data, 20.0, k.ctypes.data, 0, None, None, None, None, ct.byref(n)) == 0
    m = int(n.value)
    assert m == len(pw.generate_basis(c.recip, 20.0, k).kinetic)
    small = m - 1
    h = np.empty((small, 3), np.int32)
    a = np.empty((small, 3))
    st = lib.dftcuda_plane_wave_basis(recip.ctypes.data, 20.0, k.ctypes.data, small, h.ctypes.data, a.ctypes.data, a.ctypes.data,
                                      a.ctypes.data, ct.byref(n))
    assert st == dz.InvalidMatrixSize.status


@pytest.mark.parametrize("l", [0, 1, 2, 3, 4])
def test_projector_phi_matches_oracle(dz, l):
    rng = np.random.default_rng(7 + l)
    r = np.exp(np.linspace(math.log(1e-4), math.log(8.0), 600))
    rab = r * (math.log(8.0) - math.log(1e-4)) / 599
    beta = r ** (l + 1) * np.exp(-r * r / 1.7)
    gmax = 12.0
    tab = pseudo.RadialTable(beta, r, rab, l, gmax, n_points=512)
    q = rng.normal(scale=3.0, size=(4000, 3))
    q[0] = 0.0                                   # the origin: R(0) Y_l0 convention
    q[1] = [gmax * 1.5, 0.0, 0.0]                # beyond the table: 0
    q[2] = [gmax * (1.0 - 1e-9), 0.0, 0.0]       # in the last interval
    phi = dz.projector_phi(l, (tab.values, gmax, tab.dg), q)
    gm = np.sqrt((q * q).sum(axis=1))
    ref = np.array([4.0 * math.pi * tab.eval(gm) * pseudo.real_ylm(l, m, q[:, 0], q[:, 1], q[:, 2]) for m in range(-l, l + 1)])
    assert phi.shape == ref.shape
    assert np.abs(phi - ref).max() <= 1e-13 * np.abs(ref).max()


def test_device_kpoint_inputs_match_host(dz):
    """The resident driver's per-k inputs (basis and projector rows from the device) equal the host
    builder's: identical basis, projector rows to 1e-13."""
    import importlib

    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si8", 1)
    tables = [[system.radial_table(sp, i, 20.0) for i in range(len(sp.betas))] for sp in c.species]
    k = (0.25, 0.0, 0.125)
    a = system.kpoint_inputs(c, 20.0, k, tables=tables)
    b = system.kpoint_inputs_device(dz, c, 20.0, k, local_r=a.local_r, tables=tables)
    assert np.array_equal(a.basis.hkl, b.basis.hkl) and np.array_equal(a.basis.kinetic, b.basis.kinetic)
    for (la, da, pa), (lb, db, pb) in zip(a.species_phi, b.species_phi):
        assert la == lb and np.array_equal(da, db)
        assert np.abs(pa - pb).max() <= 1e-13 * np.abs(pa).max()
