"""The package's host-side inputs (dft-zig_b200/system.py) equal the oracle's restatement."""
import importlib

import numpy as np
import pytest

from oracle import cases

import dftzig_loader

dftzig_loader.load()
system = importlib.import_module("dftzig_b200.system")


@pytest.mark.parametrize("name,ecut,k", [("si2", 20.0, (0.25, 0.125, 0.0)), ("al4", 25.0, (0.1, 0.2, 0.3)), ("sige8", 20.0, (0.0, 0.5, 0.25))])
def test_inputs_match_oracle(name, ecut, k):
    c = system.crystal(name, 1)
    inp = system.kpoint_inputs(c, ecut, k)
    kp = cases.make_kproblem(cases.make_cell(name, 1), ecut, k)
    assert inp.dims == (kp.grid.nx, kp.grid.ny, kp.grid.nz)
    b = kp.ctx.basis
    assert (inp.basis.hkl == b.hkl).all()
    assert np.array_equal(inp.basis.kinetic, b.kinetic)
    assert np.allclose(inp.positions, np.array([a.position for a in kp.ctx.atoms]), atol=0, rtol=0)
    assert np.abs(inp.local_r - kp.ctx.local_r).max() < 1e-12 * np.abs(kp.ctx.local_r).max()
    for (l, d, phi), ns in zip(inp.species_phi, kp.ctx.nl):
        assert list(l) == list(ns.l_list)
        assert np.array_equal(d, ns.dij)
        assert np.abs(phi - ns.phi).max() < 1e-12 * np.abs(ns.phi).max()


@pytest.mark.parametrize("name,k", [("si2", (0.25, 0.125, 0.0)), ("sige8", (0.0, 0.0, 0.0))])
def test_projector_derivatives_match_oracle(name, k):
    """The host derivative projectors of the nonlocal stress equal the oracle's (oracle/stress.py,
    with the oracle's radial tables and RadialTable.eval_deriv), Gamma's q = 0 entry included."""
    from oracle import pseudo
    from oracle import stress as ost

    ecut = 20.0
    c = system.crystal(name, 1)
    kpg = system.basis(c.recip, ecut, k).kpg
    oc = cases.make_cell(name, 1)
    for sp, osp in zip(c.species, oc.species):
        host = system.projector_derivatives(sp, kpg, [system.radial_table(sp, i, ecut) for i in range(len(sp.betas))])
        tabs = pseudo.radial_tables(osp, ecut)
        _, ref = ost.projector_derivatives([l for l, _ in osp.betas], lambda b, q: tabs[b].eval(q),
                                           lambda b, q: tabs[b].eval_deriv(q), kpg)
        assert host.shape == ref.shape
        assert np.abs(host - ref).max() <= 1e-12 * np.abs(ref).max()


def test_monkhorst_pack_weights():
    k = system.monkhorst_pack((2, 2, 2))
    assert len(k) == 8 and abs(sum(w for _, w in k) - 1.0) < 1e-15
    k4 = system.monkhorst_pack((4, 4, 4))
    assert abs(sum(w for _, w in k4) - 1.0) < 1e-15 and len(k4) == 36


@pytest.mark.parametrize("name,ecut,box", [("si2", 20.0, (20, 20, 20)), ("si2", 30.0, (24, 24, 24)), ("al4", 25.0, (27, 27, 27)),
                                           ("si64", 30.0, (75, 75, 75)), ("si216", 25.0, (108, 108, 108)),
                                           ("sige8", 20.0, (36, 32, 32)), ("sival", 25.0, (108, 100, 72))])
def test_every_cell_box_has_a_register_fft_split(name, ecut, box):
    """The FFT box of each cell the tests and the bench run (fft_box: 2-3-5-smooth, >= 2 G_max + 1)
    is one the fused register-FFT passes implement (DFTCUDA_FOUR_STEP_LENGTHS in csrc/fft_reg.cuh),
    so none of them falls back to the generic passes."""
    import os
    import re

    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dft-zig_b200", "csrc", "fft_reg.cuh")).read()
    macro = src[src.index("#define DFTCUDA_FOUR_STEP_LENGTHS"):].split("\n\n")[0]
    lengths = {int(v) for v in re.findall(r"X\((\d+)\)", macro)}
    c = system.crystal(name, 1)
    dims = system.fft_box(ecut, c.recip)
    assert tuple(dims) == box
    assert set(dims) <= lengths
