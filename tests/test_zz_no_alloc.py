"""The allocation-free band-density entry point (dftcuda_accumulate_density_noalloc).

It exists for callers that cannot call cudaMalloc -- a framework that owns all device memory through
its own pool, or a loop that must not take the device-wide synchronisation an allocation can cause.
It keeps its scratch in a fixed 48 MiB array of the library's device image.  This file is collected
last so that, if it fails, a run that stops at the first failure has already run every other test.
It is called here through the C ABI (ctypes) and compared with dftcuda_accumulate_density on two
calls in a row, which also shows that the scratch's leftover contents from one call do not leak
into the next; FP64 and FP32 contexts, and a call with more bands than one pass of the scratch
holds (so the columns go through it in several chunks).
"""
import ctypes as ct

import numpy as np
import pytest

from tests.helpers import kproblem, make_context, random_block

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 5e-5}  # relative: the FP64 density bar, and the FP32 FFT-pass bar
SCRATCH = 48 << 20


def _noalloc(dz, kc, v_dev, w_dev, rho_dev, nbands):
    lib = dz.load_library()
    return lib.dftcuda_accumulate_density_noalloc(kc.handle, ct.c_void_p(v_dev.data_ptr()), kc.n, nbands, ct.c_void_p(w_dev.data_ptr()), ct.c_void_p(rho_dev.data_ptr()))


def _case(dz, torch, name, ecut, k, nb, seed, precision=0):
    kp = kproblem(name, ecut, k)
    kc = make_context(dz, kp, precision)
    v = random_block(kp.ctx.n, nb, seed)
    w = np.linspace(2.0, -0.5, nb)  # includes zero and negative weights, which contribute nothing
    rho_ref = np.full(kp.grid.count, 0.125)
    kc.accumulate_band_density(v, w, rho_ref)
    v_dev = torch.from_numpy(v).cuda()
    w_dev = torch.from_numpy(w).cuda()
    rho_dev = torch.full((kp.grid.count,), 0.125, dtype=torch.float64, device="cuda")
    # The entry point orders itself after the legacy default stream; synchronising here as well
    # keeps the inputs' uploads complete whatever stream torch used for them.
    torch.cuda.synchronize()
    status = _noalloc(dz, kc, v_dev, w_dev, rho_dev, nb)
    assert status == 0, dz.load_library().dftcuda_last_error_message()
    got = rho_dev.cpu().numpy()
    assert np.abs(got - rho_ref).max() < TOL[precision] * np.abs(rho_ref).max()
    return kc, kp


def test_noalloc_density_matches_existing_entry_point_twice(dz):
    import torch

    # first call: Si8, 32^3 box, 40 bands; second call: Si2, 20^3 box, 7 bands, on a different
    # context, so the second call reads a scratch array the first left filled with other data.
    kc1, _ = _case(dz, torch, "si8", 20.0, (0.25, 0.0, 0.0), 40, 3)
    kc2, _ = _case(dz, torch, "si2", 20.0, (0.25, 0.125, 0.0), 7, 4)
    kc1.close()
    kc2.close()


def test_noalloc_density_fp32_context(dz):
    import torch

    kc1, _ = _case(dz, torch, "si8", 20.0, (0.0, 0.25, 0.0), 24, 5, precision=1)
    kc2, _ = _case(dz, torch, "si2", 20.0, (0.125, 0.0, 0.25), 9, 6, precision=1)
    kc1.close()
    kc2.close()


def test_noalloc_density_in_several_chunks(dz):
    import torch

    # 400 Si8 bands need more y-z planes than one pass of the scratch holds, so the columns run in
    # chunks (weights read at the chunk's offset); the result still equals the one-call density.
    kc, kp = _case(dz, torch, "si8", 20.0, (0.125, 0.125, 0.0), 400, 7)
    n_act = len(np.unique(kp.ctx.basis.hkl[:, 0]))
    per_col = 16 * n_act * kp.grid.ny * kp.grid.nz
    assert 400 * per_col > SCRATCH - 4096 * 8, "case must not fit one pass of the scratch"
    kc.close()


def test_noalloc_density_rejects_too_many_bands_and_host_pointers(dz):
    import torch

    kp = kproblem("si2", 20.0)
    kc = make_context(dz, kp)
    lib = dz.load_library()
    nb = 4097  # DFTCUDA_NOALLOC_MAX_BANDS + 1
    v_dev = torch.zeros((nb, kp.ctx.n), dtype=torch.complex128, device="cuda")
    w_dev = torch.ones(nb, dtype=torch.float64, device="cuda")
    rho_dev = torch.zeros(kp.grid.count, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(dz, kc, v_dev, w_dev, rho_dev, nb) == -7
    assert b"DFTCUDA_NOALLOC_MAX_BANDS" in lib.dftcuda_last_error_message()
    host_rho = np.zeros(kp.grid.count)
    st = lib.dftcuda_accumulate_density_noalloc(kc.handle, ct.c_void_p(v_dev.data_ptr()), kc.n, 1, ct.c_void_p(w_dev.data_ptr()), host_rho.ctypes.data)
    assert st == -6
    kc.close()


def test_plane_beyond_shared_memory_is_rejected(dz):
    """A y-z plane of 128 x 128 FP64 complex values (256 KB) does not fit one CTA's shared memory.
    Context creation already refuses it (Unsupported), so no entry point, the allocation-free
    density included (which checks again), can launch an oversized plane; the FP32 context of the
    same box (128 KB planes) is accepted and its allocation-free density runs."""
    import torch

    dims = (20, 128, 128)
    hkl = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.int32)
    kin = np.array([0.0, 1.0, 1.0, 1.0])
    gcart = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    with pytest.raises(dz.Unsupported):
        dz.KpointContext(*dims, 1000.0, hkl, kin, gcart, 0)
    kc = dz.KpointContext(*dims, 1000.0, hkl, kin, gcart, 1)
    v = torch.ones((2, 4), dtype=torch.complex128, device="cuda")
    w = torch.ones(2, dtype=torch.float64, device="cuda")
    rho = torch.zeros(dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    kc.accumulate_band_density_noalloc(v, w, rho)
    torch.cuda.synchronize()
    # Parseval: the density integrates to sum_b w_b sum_G |c_G|^2 = 2 bands x 4 plane waves
    assert abs(float(rho.sum()) * 1000.0 / rho.numel() - 8.0) < 1e-4
    kc.close()
