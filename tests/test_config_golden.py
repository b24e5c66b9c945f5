"""The committed config-size oracle fixtures (tests/golden/config_parity.json) are what the oracle
computes: the two cheap ones (Si2 4x4x4 SCF, Al4 three k-points) are recomputed here on the CPU and
must match to the last digits the GPU parity tests rely on."""
import json
import os

import numpy as np

from tests.golden import make_config_parity as mk

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_parity.json")))


def _same(a, b):
    assert a["converged"] and b["converged"]
    assert abs(a["energy_per_atom"] - b["energy_per_atom"]) < 1e-12
    for x, y in zip(a["eigenvalues"], b["eigenvalues"]):
        assert np.abs(np.asarray(x) - np.asarray(y)).max() < 1e-11


def test_si2_444_fixture():
    _same(mk.si2_444_scf(), GOLDEN["si2_444_scf"])


def test_al4_three_k_fixture():
    _same(mk.al4_888_three_k(), GOLDEN["al4_888_three_k"])


def test_si64_fixture_shape():
    g = GOLDEN["si64_gamma_davidson"]
    assert g["nbands"] == 160 and len(g["eigenvalues"]) == 160 and g["dims"] == [75, 75, 75]
    assert np.all(np.diff(g["eigenvalues"]) >= 0)
