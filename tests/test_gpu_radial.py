"""Radial projector tables on the device (dftcuda_radial_table) against the oracle's RadialTable
(oracle/pseudo.py, a restatement of pseudopotential/nonlocal.zig:8-21, 59-71, 250-338) and the
host table builder; l = 0..4 exercises the closed forms, the small-argument series and the
downward recursion."""
import importlib
import math

import numpy as np
import pytest

from oracle import pseudo as ps

pytestmark = pytest.mark.gpu


def _mesh(n=421):
    # logarithmic mesh like a UPF file: r_i = exp(xmin + i dx) / z, rab_i = r_i dx
    dx = 0.0125
    r = np.exp(-7.0 + dx * np.arange(n)) / 14.0
    return r, r * dx


@pytest.mark.parametrize("l", [0, 1, 2, 3, 4])
def test_radial_table_matches_oracle(dz, l):
    r, rab = _mesh()
    rng = np.random.default_rng(10 + l)
    rbeta = r ** (l + 1) * np.exp(-r * r / 1.3) * (1.0 + 0.2 * rng.normal(size=r.size))
    gmax = 1.5 * math.sqrt(2.0 * 25.0)
    npts = 257 if l >= 2 else 2048  # the oracle's Miller recursion runs per element in Python
    ref = ps.RadialTable(rbeta, r, rab, l, gmax, npts).values
    got, gm, dq = dz.radial_table(l, r, rbeta, rab, gmax, npts)
    assert gm == gmax and abs(dq - gmax / (npts - 1)) < 1e-15
    assert np.abs(got - ref).max() <= 1e-12 * max(1e-300, np.abs(ref).max())


def test_radial_table_short_mesh_and_errors(dz):
    # fewer than 10 points: plain weights
    r = np.linspace(0.1, 2.0, 7)
    rab = np.full(7, r[1] - r[0])
    rbeta = np.exp(-r)
    ref = ps.RadialTable(rbeta, r, rab, 1, 4.0, 16).values
    got, _, _ = dz.radial_table(1, r, rbeta, rab, 4.0, 16)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    with pytest.raises(Exception):
        dz.radial_table(0, r, rbeta, rab, 4.0, 1)
    with pytest.raises(Exception):
        dz.radial_table(0, r, rbeta, rab, -1.0, 16)


def test_radial_table_matches_host_builder(dz):
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si2")
    sp = c.species[0]
    for b, (l, beta) in enumerate(sp.betas):
        host = system.radial_table(sp, b, 20.0)
        dev = dz.radial_table(l, sp.r, beta, sp.rab, host[1])
        assert np.abs(dev[0] - host[0]).max() <= 1e-12 * np.abs(host[0]).max()
