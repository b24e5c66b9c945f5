"""Density symmetrisation on the device (dftcuda_symmetrize_density) against the oracle's restatement
of symmetrize_density (oracle/symmetry.py; scf/density_symmetry.zig:27-94), with the operations of
diamond cells from the oracle's space-group search."""
import importlib
import math

import numpy as np
import pytest

from oracle import symmetry as sy

pytestmark = pytest.mark.gpu


def _case(name):
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal(name)
    cell = np.asarray(c.cell, dtype=np.float64)
    frac = np.asarray(c.positions, dtype=np.float64) @ np.linalg.inv(cell)
    recip = 2 * math.pi * np.linalg.inv(cell).T
    return cell, recip, sy.symmetry_ops(cell, frac, c.atom_species)


@pytest.mark.parametrize("name,dims", [("si2", (16, 16, 16)), ("si2", (12, 10, 9)), ("si8", (24, 24, 24))])
def test_symmetrize_matches_oracle(dz, name, dims):
    import torch

    cell, recip, ops = _case(name)
    n = dims[0] * dims[1] * dims[2]
    rho = 0.05 + 0.01 * np.random.default_rng(n).random(n)
    ref = sy.symmetrize_density(rho, dims, ops)
    pc = dz.PotentialContext(dims, abs(np.linalg.det(cell)), recip, history=1)
    try:
        host = pc.symmetrize(rho.copy(), ops)  # host array, in place
        assert np.abs(host - ref).max() <= 1e-12 * np.abs(ref).max()
        dev = torch.from_numpy(rho.copy()).cuda()
        pc.symmetrize(dev, ops)  # device tensor, in place
        assert np.abs(dev.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
        # a second pass changes nothing (up to rounding) when no rotated index wraps
        if name == "si8":
            again = pc.symmetrize(host.copy(), ops)
            assert np.abs(again - host).max() <= 1e-12 * np.abs(host).max()
    finally:
        pc.close()


def test_symmetrize_identity_and_errors(dz):
    cell, recip, ops = _case("si2")
    dims = (8, 8, 8)
    rho = np.random.default_rng(5).random(512)
    pc = dz.PotentialContext(dims, abs(np.linalg.det(cell)), recip, history=1)
    try:
        ident = [(np.eye(3, dtype=np.int32), np.zeros(3))]
        assert np.array_equal(pc.symmetrize(rho.copy(), ident), rho)
        assert np.array_equal(pc.symmetrize(rho.copy(), []), rho)
        with pytest.raises(Exception):
            pc.symmetrize(rho.copy(), ops * 5)  # 240 operations: above the 192 the entry point takes
        bad = [(o[1], np.array([np.nan, 0.0, 0.0])) for o in ops[:2]]
        with pytest.raises(Exception):
            pc.symmetrize(rho.copy(), bad)
    finally:
        pc.close()
