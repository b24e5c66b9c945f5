"""Band density rho += w |psi(r)|^2 / Omega on the GPU against the oracle (kpoint/density.zig:444-474)."""
import numpy as np
import pytest

from oracle import density as odens
from tests.helpers import kproblem, make_context, random_block

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,ecut,k", [("si2", 20.0, (0.25, 0.0, 0.0)), ("sige8", 20.0, (0.0, 0.0, 0.0)), ("si64", 30.0, (0.0, 0.0, 0.0))])
def test_density_matches_oracle(dz, name, ecut, k):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp)
    nb = 6
    v = random_block(kp.ctx.n, nb, 2)
    w = np.array([2.0, 2.0, 1.0, 0.0, -1.0, 0.5])  # zero / negative weights are skipped
    rho = np.full(kp.grid.count, 0.25)
    kc.accumulate_band_density(v, w, rho)
    ref = 0.25 + odens.accumulate_density(kp.grid, kp.ctx.map, v, w, 1.0 / kp.grid.volume)
    assert np.abs(rho - ref).max() < 1e-12 * np.abs(ref).max()
    kc.close()


def test_density_device_pointers(dz):
    import torch

    kp = kproblem("si2", 20.0)
    kc = make_context(dz, kp)
    v = random_block(kp.ctx.n, 3, 8)
    w = np.array([2.0, 1.0, 0.5])
    rho_h = np.zeros(kp.grid.count)
    kc.accumulate_band_density(v, w, rho_h)
    rho_d = torch.zeros(kp.grid.count, dtype=torch.float64, device="cuda")
    kc.accumulate_band_density(torch.from_numpy(v).cuda(), w, rho_d)
    assert np.abs(rho_d.cpu().numpy() - rho_h).max() < 1e-14 * np.abs(rho_h).max()
    kc.close()
