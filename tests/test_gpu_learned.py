"""Learned preconditioner on the GPU: the CUDA forward/backward kernels against the CPU oracle
(oracle/learned.py, itself checked against finite differences), training reduces the loss, and every
preconditioner kind converges the Davidson solver to the same eigenvalues."""
import numpy as np
import pytest

from oracle import learned
from tests.helpers import kproblem, make_context

pytestmark = pytest.mark.gpu


def test_loss_and_gradient_match_oracle(dz):
    off, feat, cc, w, dnorm = learned.random_problem(nbands=9, per_band=(100, 300), seed=5)
    p = learned.init_params(seed=3)
    # the GPU computes in FP32 from FP32 inputs: give the oracle the same rounded inputs
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    cc32 = f32(cc.real) + 1j * f32(cc.imag)
    L_ref, g_ref = learned.loss_grad(f32(p), off, f32(feat), cc32, f32(w), f32(dnorm))
    L, g = dz.precond_mlp_loss_grad(p, off, feat, cc, w, dnorm)
    assert abs(L - L_ref) < 1e-5
    assert np.abs(g - g_ref).max() < 2e-4 * np.abs(g_ref).max()


def test_training_reduces_loss(dz):
    off, feat, cc, w, dnorm = learned.random_problem(nbands=24, per_band=(200, 400), seed=6)
    p0 = learned.init_params(seed=4)
    p, hist = dz.precond_mlp_train(p0, off, feat, cc, w, dnorm, steps=200, lr=3e-3)
    assert hist[-1] < 0.8 * hist[0]
    L_final, _ = dz.precond_mlp_loss_grad(p, off, feat, cc, w, dnorm)
    assert L_final <= hist[-1] + 1e-6


@pytest.mark.parametrize("kind", ["tpa", "mlp"])
def test_preconditioners_reach_the_same_eigenvalues(dz, kind):
    kp = kproblem("si8", 12.0, (0.25, 0.0, 0.0))
    diag = kp.ctx.basis.kinetic
    opts = dz.Options(max_iter=200, tol=1e-8)
    kc = make_context(dz, kp)
    ref = kc.hermitian_eigen_decomp_iterative(diag, 16, opts)
    if kind == "tpa":
        kc.set_preconditioner(dz.PRECOND_TPA)
    else:
        kc.set_preconditioner(dz.PRECOND_MLP, learned.init_params(seed=7).astype(np.float32))
    alt = kc.hermitian_eigen_decomp_iterative(diag, 16, opts)
    kc.close()
    assert ref.converged and alt.converged
    assert np.abs(ref.values - alt.values).max() < 1e-7


def test_preconditioner_argument_errors(dz):
    kp = kproblem("si2", 10.0)
    kc = make_context(dz, kp)
    with pytest.raises(dz.InvalidArgument):
        kc.set_preconditioner(dz.PRECOND_MLP, np.zeros(10, np.float32))
    with pytest.raises(dz.InvalidArgument):
        kc.set_preconditioner(7)
    kc.close()


# ---- Fourier neural operator ----------------------------------------------------------------------


def _fno_samples(seed):
    rng = np.random.default_rng(seed)
    out = []
    for dims in ((16, 16, 18), (20, 16, 16)):
        n = int(np.prod(dims))
        u = rng.random((2, n))
        out.append((dims, u, 0.1 * rng.normal(size=n)))
    return out


def test_fno_forward_and_gradient_match_autograd_oracle(dz):
    samples = _fno_samples(1)
    p = learned.fno_init_params(2)
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    L_ref, g_ref = learned.fno_loss_grad(f32(p), [(d, f32(u), f32(t)) for d, u, t in samples])
    L, g = dz.fno_loss_grad(p, samples)
    assert abs(L - L_ref) < 1e-5 * max(1.0, L_ref)
    assert np.abs(g - g_ref).max() < 1e-3 * np.abs(g_ref).max()
    import torch
    d0 = learned.fno_forward_torch(torch.tensor(f32(p)), f32(samples[0][1]), samples[0][0]).numpy()
    out = dz.fno_forward(p, samples[0][1], samples[0][0])
    assert np.abs(out - d0).max() < 1e-4 * max(1.0, np.abs(d0).max())


def test_fno_training_reduces_loss(dz):
    samples = _fno_samples(3)
    p0 = learned.fno_init_params(4)
    p, hist = dz.fno_train(p0, samples, steps=60, lr=2e-3)
    assert hist[-1] < 0.7 * hist[0]


# ---- the shipped trained weights on held-out cells ------------------------------------------------


@pytest.mark.parametrize("seed", [1290, 1291])
def test_trained_preconditioner_gain(dz, seed):
    """The committed MLP preconditioner on held-out cells of its training family (Si cells of 8 to 64
    atoms, strained and displaced): converges to the reference eigenvalues in far fewer H
    applications than the reference diagonal, and in fewer than Teter-Payne-Allan, the form it
    refines -- the test fails if the network stops beating its base."""
    import importlib

    learn = importlib.import_module("dftzig_b200.learn")
    system = importlib.import_module("dftzig_b200.system")
    params = learn.load_precond_weights()
    c = system.crystal("sitrain", seed)
    nb = int(round(c.nelec / 2))
    inp = system.kpoint_inputs(c, 25.0, (0.0, 0.0, 0.0))
    out = {}
    for kind in (dz.PRECOND_REFERENCE, dz.PRECOND_TPA, dz.PRECOND_MLP):
        kc = learn._context(dz, inp)
        kc.set_preconditioner(kind, params if kind == dz.PRECOND_MLP else None)
        out[kind] = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, nb, dz.Options(max_iter=400, tol=1e-6))
        kc.close()
    ref, tpa, mlp = out[dz.PRECOND_REFERENCE], out[dz.PRECOND_TPA], out[dz.PRECOND_MLP]
    assert ref.converged and tpa.converged and mlp.converged
    assert np.abs(mlp.values - ref.values).max() < 1e-7
    assert mlp.h_applies < 0.5 * ref.h_applies
    assert mlp.h_applies < tpa.h_applies


_INFER_SCRIPT = """
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
import importlib
import dftzig_loader
dz = dftzig_loader.load()
learn = importlib.import_module("dftzig_b200.learn")
system = importlib.import_module("dftzig_b200.system")
c = system.crystal("sitrain", 1290)
nb = int(round(c.nelec / 2))
inp = system.kpoint_inputs(c, 25.0, (0.0, 0.0, 0.0))
kc = learn._context(dz, inp)
kc.set_preconditioner(dz.PRECOND_MLP, learn.load_precond_weights())
r = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, nb, dz.Options(max_iter=400, tol=1e-6))
kc.close()
print(json.dumps({{"values": list(map(float, r.values)), "h_applies": int(r.h_applies), "converged": bool(r.converged)}}))
"""


def test_mlp_table_inference_matches_tensor_core_form():
    """The default inference interpolates a table of the FP32 network (|dz| <= 5e-5); the tensor-core
    form (DFTCUDA_MLP_INFER=tc) evaluates the network per entry with TF32 operands.  Both steer the
    Davidson solve of a held-out cell to the same eigenvalues in about the same number of H
    applications."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for mode in ("table", "tc"):
        env = dict(os.environ)
        env.pop("DFTCUDA_MLP_INFER", None)
        if mode == "tc":
            env["DFTCUDA_MLP_INFER"] = "tc"
        r = subprocess.run([sys.executable, "-c", _INFER_SCRIPT.format(root=root)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[mode] = json.loads(r.stdout.strip().splitlines()[-1])
    a, b = out["table"], out["tc"]
    assert a["converged"] and b["converged"]
    assert np.abs(np.array(a["values"]) - np.array(b["values"])).max() < 1e-7
    assert abs(a["h_applies"] - b["h_applies"]) <= 0.05 * b["h_applies"]


def test_trained_fno_start_beats_atomic_superposition(dz):
    """The committed FNO on a held-out SiGe8 cell: its first density is far closer to the converged
    SCF density than the atomic superposition it starts from."""
    import importlib

    learn = importlib.import_module("dftzig_b200.learn")
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("sige8", 2490)
    ecut = 20.0
    dims, u, rho_at, mean = learn.fno_input(c, ecut)
    rho_fno = learn.fno_initial_density(dz, learn.load_fno_weights(), c, ecut)
    b = scf.GpuBackend(dz)
    r = scf.run_scf(c, scf.ScfParams(ecut=ecut, kmesh=(2, 2, 2), nbands=20, convergence=1e-7, smearing=learn.FNO_SMEARING, max_iter=80), b)
    b.close()
    assert r.converged
    rho_atomic = rho_at * (c.nelec / (rho_at.mean() * c.volume))
    err_fno = np.sqrt(np.mean((rho_fno - r.rho) ** 2))
    err_at = np.sqrt(np.mean((rho_atomic - r.rho) ** 2))
    assert err_fno < 0.2 * err_at


def test_trained_preconditioner_scf_gain(dz):
    """The committed MLP preconditioner inside a whole SCF run (warm-started Davidson every step, the
    reference's mixing and eigensolver defaults) on a held-out 32-atom cell of its training family:
    the same converged energy in fewer H applications than Teter-Payne-Allan."""
    import importlib

    learn = importlib.import_module("dftzig_b200.learn")
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("sitrain", 1207)
    assert len(c.atom_species) == 32
    nb = int(round(c.nelec / 2.0)) + 8
    out = {}
    for key, pre in (("tpa", (dz.PRECOND_TPA, None)), ("mlp", (dz.PRECOND_MLP, learn.load_precond_weights()))):
        b = scf.GpuBackend(dz, "fp64", precond=pre, resident=True)
        r = scf.run_scf(c, scf.ScfParams(ecut=25.0, kmesh=(1, 1, 1), nbands=nb, convergence=1e-7, max_iter=60), b)
        b.close()
        out[key] = (r, sum(s[2] for s in b.solves))
    (rt, ht), (rm, hm) = out["tpa"], out["mlp"]
    assert rt.converged and rm.converged
    assert abs(rt.energy_per_atom - rm.energy_per_atom) < 1e-6
    assert hm < ht
