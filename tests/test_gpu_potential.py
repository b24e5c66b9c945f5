"""The device potential build and Pulay mixing (dftcuda_pctx_*, csrc/potential.cu) against the oracle
(oracle/potential.py): host and device buffers, odd and even boxes, a triclinic cell."""
import importlib
import math

import numpy as np
import pytest
import torch

from oracle import potential as op

pytestmark = pytest.mark.gpu

RECIP = np.array([[0.61, 0.05, 0.0], [0.02, 0.57, 0.04], [0.0, -0.03, 0.66]])
VOL = (2 * math.pi) ** 3 / abs(np.linalg.det(RECIP))
BOXES = [(12, 10, 9), (24, 24, 24), (45, 40, 36)]


def _rho(dims, seed):
    rng = np.random.default_rng(seed)
    n = dims[0] * dims[1] * dims[2]
    x = 0.01 + 0.08 * rng.random(n)
    x[:5] = 0.0  # points at and below the LDA cut
    return x


@pytest.mark.parametrize("dims", BOXES)
def test_hxc_potential_matches_oracle(dz, dims):
    pc = dz.PotentialContext(dims, VOL, RECIP, history=4)
    try:
        rho = _rho(dims, 1)
        v_in = op.to_g(np.sin(np.arange(rho.size) * 0.003), dims)
        ref, e_h, e_xc, ivr = op.hxc_potential(rho, dims, RECIP, VOL, v_in)
        scale = np.abs(ref).max()
        # host arrays
        v, t = pc.hxc(rho, v_in)
        assert np.abs(v - ref).max() < 1e-12 * scale
        assert abs(t["e_hartree"] - e_h) < 1e-11 * abs(e_h)
        assert abs(t["e_xc"] - e_xc) < 1e-11 * abs(e_xc)
        assert abs(t["int_vin_rho"] - ivr) < 1e-11 * max(abs(ivr), 1e-3)
        # device tensors, no v_in
        vd, td = pc.hxc(torch.from_numpy(rho).cuda())
        assert vd.is_cuda
        assert np.abs(vd.cpu().numpy() - ref).max() < 1e-12 * scale
        assert td["int_vin_rho"] == 0.0 and abs(td["e_hartree"] - e_h) < 1e-11 * abs(e_h)
    finally:
        pc.close()


def test_potential_real_matches_oracle(dz):
    dims = BOXES[2]
    pc = dz.PotentialContext(dims, VOL, RECIP, history=2)
    try:
        rng = np.random.default_rng(2)
        v = op.to_g(rng.normal(size=dims[0] * dims[1] * dims[2]), dims)
        vloc = rng.normal(size=v.size)
        ref = op.potential_real(v, vloc, dims)
        out = pc.real(v, vloc)
        assert np.abs(out - ref).max() < 1e-12 * np.abs(ref).max()
        outd = pc.real(torch.from_numpy(v).cuda())
        assert np.abs(outd.cpu().numpy() - op.potential_real(v, None, dims)).max() < 1e-12 * np.abs(ref).max()
    finally:
        pc.close()


@pytest.mark.parametrize("on_device", [False, True], ids=["host", "device"])
def test_pulay_mix_matches_oracle(dz, on_device):
    """Eight steps with a history of four on a linear fixed point x = b + (1 - A) x in 2000 dims,
    then a reset: the device history, overlaps and DIIS weights follow the oracle's device form.
    The operator's spectrum is wide (0.3 .. 1.2): with a narrow one the residuals are nearly
    collinear and the DIIS weights amplify summation-order rounding to 1e-9 (the oracle against
    itself with its dot products summed in another order)."""
    rng = np.random.default_rng(5)
    n = 2000
    A = 0.3 + 0.9 * rng.random(n)  # a diagonal operator: residual b - A x
    b = rng.normal(size=n)
    pc = dz.PotentialContext((4, 4, 4), 1.0, np.eye(3), history=4)
    try:
        mo = op.Pulay(4, device_form=True)
        x_ref = np.zeros(n)
        x = torch.zeros(n, dtype=torch.float64, device="cuda") if on_device else np.zeros(n)
        for it in range(10):
            if it == 8:
                pc.reset()
                mo = op.Pulay(4, device_form=True)
            r_ref = b - A * x_ref
            x_ref = mo.mix(x_ref, r_ref, 0.5)
            xh = x.cpu().numpy() if on_device else x
            r = b - A * xh
            if on_device:
                pc.pulay_mix(x, torch.from_numpy(r).cuda(), 0.5)
            else:
                pc.pulay_mix(x, r, 0.5)
            got = x.cpu().numpy() if on_device else x
            assert np.abs(got - x_ref).max() < 1e-10 * max(1.0, np.abs(x_ref).max()), it
        assert np.linalg.norm(b - A * x_ref) < 0.1 * np.linalg.norm(b)
    finally:
        pc.close()


def test_pulay_mix_rejects_missing_history(dz):
    pc = dz.PotentialContext((4, 4, 4), 1.0, np.eye(3), history=0)
    try:
        with pytest.raises(dz.DftCudaError):
            pc.pulay_mix(np.zeros(8), np.zeros(8), 0.5)
    finally:
        pc.close()


def test_ionic_potential_matches_oracle(dz):
    """Two species with all four GTH coefficients, 37 atoms in a triclinic cell, an odd box, with and
    without the |G|^2 cut; V(G) and V_loc(r) to host and device buffers."""
    dims = (27, 24, 25)
    rng = np.random.default_rng(11)
    cell = np.linalg.inv(RECIP).T * 2 * math.pi
    pos = rng.random((37, 3)) @ cell
    sp = rng.integers(0, 2, 37).astype(np.int32)
    gth = [[4.0, 0.44, -7.3, 1.1, -0.2, 0.03], [3.0, 0.5, -6.0, 0.0, 0.4, 0.0]]
    pc = dz.PotentialContext(dims, VOL, RECIP, history=1)
    try:
        for g2max in (0.0, 30.0):
            ref_g, ref_r = op.ionic_potential(gth, sp, pos, dims, RECIP, VOL, g2max)
            vg, vr = pc.ionic(gth, sp, pos, g2max)
            assert np.abs(vg - ref_g).max() < 1e-12 * np.abs(ref_g).max()
            assert np.abs(vr - ref_r).max() < 1e-11 * np.abs(ref_r).max()
            vgd, vrd = pc.ionic(gth, sp, pos, g2max, device=True)
            assert vrd.is_cuda and np.abs(vrd.cpu().numpy() - ref_r).max() < 1e-11 * np.abs(ref_r).max()
        with pytest.raises(dz.DftCudaError):
            pc.ionic(gth, np.array([0, 2], dtype=np.int32), pos[:2])
    finally:
        pc.close()


def test_ionic_potential_radial_matches_oracle(dz):
    """The radial-mesh form (dftcuda_ionic_potential_radial: the reference's short-range form factor
    at every |G| of the box): two species with different meshes, 37 atoms in a triclinic cell, an odd
    box, with and without the |G|^2 cut."""
    from oracle import pseudo

    system = importlib.import_module("dftzig_b200.system")
    dims = (27, 24, 25)
    rng = np.random.default_rng(12)
    cell = np.linalg.inv(RECIP).T * 2 * math.pi
    pos = rng.random((37, 3)) @ cell
    sp = rng.integers(0, 2, 37).astype(np.int32)
    si, al = system.species("Si"), system.species("Al")
    meshes = [si.mesh, (al.r[::2], al.rab[::2] * 2.0, al.vloc[::2], al.z_val)]  # a coarser second mesh
    pc = dz.PotentialContext(dims, VOL, RECIP, history=1)
    try:
        for g2max in (0.0, 30.0):
            ref_g, _ = pseudo.ionic_potential_radial(meshes, sp, pos, dims, RECIP, VOL, g2max)
            ref_r = op.to_r(ref_g, dims)
            vg, vr = pc.ionic_radial(meshes, sp, pos, g2max)
            assert np.abs(vg - ref_g).max() < 1e-12 * np.abs(ref_g).max()
            assert np.abs(vr - ref_r).max() < 1e-11 * np.abs(ref_r).max()
    finally:
        pc.close()


@pytest.mark.parametrize("dims", [(12, 10, 9), (24, 24, 24)])
def test_pbe_potential_matches_oracle(dz, dims):
    """PBE through the device: gradient by three inverse FFTs, the point functional, the divergence by
    FFTs; V_hxc(G) and the energy terms against the oracle's assembly."""
    pc = dz.PotentialContext(dims, VOL, RECIP, history=1, functional="pbe")
    try:
        rng = np.random.default_rng(3)
        N = dims[0] * dims[1] * dims[2]
        g2 = op.g2_table(dims, RECIP)
        rho = 0.03 + 0.01 * op.to_r(np.where(g2 < 2.0, op.to_g(rng.normal(size=N), dims), 0.0), dims)
        v_in = op.to_g(np.cos(np.arange(N) * 0.01), dims)
        ref, e_h, e_xc, ivr = op.hxc_potential(rho, dims, RECIP, VOL, v_in, functional="pbe")
        v, t = pc.hxc(rho, v_in)
        assert np.abs(v - ref).max() < 1e-11 * np.abs(ref).max()
        assert abs(t["e_xc"] - e_xc) < 1e-11 * abs(e_xc)
        assert abs(t["e_hartree"] - e_h) < 1e-11 * abs(e_h)
        # the gradient term matters: PBE and LDA potentials differ
        lda, *_ = op.hxc_potential(rho, dims, RECIP, VOL)
        assert np.abs(ref - lda).max() > 1e-4 * np.abs(ref).max()
    finally:
        pc.close()
