"""Learned components: data generation, GPU training and evaluation.

Learned preconditioner (``precond``): a per-plane-wave MLP that refines the Teter-Payne-Allan
diagonal of the Davidson correction step (m = K_TPA(x) exp(z_theta); the reference's own form is
r / (|k+G|^2 - lambda), lobpcg/common.zig:214-226).  Training pairs come from TPA-preconditioned
runs of the device solver on 200 seeded Si cells of 8 to 64 atoms (``sitrain``: supercells of the
cubic cell with strain and displacements; the strained Si8 set ``si8d`` of the first weights stays
selectable): the solver is deterministic (LCG start, serial.zig:75-95), so the run stopped after t
iterations reproduces the Ritz vectors psi_b^t of the full run; the target is the correction from
psi_b^t to its converged eigenspace.  The trained network is judged against TPA on the Si216 cell:
Davidson iterations, H applications and wall time to the same residual (evaluate_si216).  The network is trained on the GPU by
the library's own CUDA forward/backward kernels (dftcuda_precond_mlp_train, Adam).

Learned first density (``fno``): a Fourier neural operator (csrc/fno.cu) maps the superposition of
atomic densities of a cell (build_atomic_density, scf/core_density.zig:128-183; two channels, Si-like
and Ge-like) to the converged SCF density minus that superposition.  Targets come from plain SCF
runs (flat start, the reference default, run_state.zig:98-115) on seeded SiGe8 cells; training runs
on the GPU with the library's own FNO forward/backward kernels.  The learned start is
rho0 = rho_atomic + mean * FNO(u), clipped positive and renormalised to N_e.

Usage (the package directory is registered as ``dftzig_b200`` by dftzig_loader):
    python -c "import dftzig_loader, importlib; dftzig_loader.load(); importlib.import_module('dftzig_b200.learn').main()" precond
    python -c "...same..." fno
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import scf as scfm
from . import system as sysm

WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
PRECOND_WEIGHTS = os.path.join(WEIGHTS_DIR, "precond_mlp.npz")
FNO_WEIGHTS = os.path.join(WEIGHTS_DIR, "fno_density.npz")


def _context(dz, inp, precision=0):
    kc = dz.KpointContext(*inp.dims, inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, precision)
    kc.set_vloc(inp.local_r)
    kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
    return kc


def _features(kin, ekin, rabs, rms, t):
    x = kin / max(ekin, 1e-6)
    return np.stack([np.log(x + 0.05), np.log(rabs / max(rms, 1e-300) + 1e-6), np.full_like(x, min(t / 20.0, 2.0))], axis=1)


def precond_samples(dz, cells, ecut: float, nbands, t_max: int = 20, kfrac=(0.0, 0.0, 0.0), cluster_tol: float = 1e-4,
                    min_overlap: float = 0.5, t_list=None, bands_per_t=None, seed: int = 0):
    """Residual -> correction samples along Davidson trajectories preconditioned by TPA (the form
    the network refines).  Target of band b at iteration t: delta_b = (1 - Psi Psi^H) y, y the
    normalised projection of psi_b^t on the converged eigenspace of its group of (near-)degenerate
    bands (gaps < cluster_tol Ry), kept when that projection has norm >= min_overlap, and Psi all nb
    Ritz vectors of iteration t: the part of the correction that the subspace does not hold yet
    (whatever lies in span(Psi) the Rayleigh-Ritz step finds without a new direction).
    nbands: a number, or a function of the cell (e.g. its occupied bands); t_list: the iterations
    sampled (default 1..t_max); bands_per_t: keep at most this many bands per (cell, t), drawn with
    a seeded generator (bounds the data of large cells)."""
    off = [0]
    feats, ccs, ws, dns, kins, lams = [], [], [], [], [], []
    rng = np.random.default_rng(seed)
    for c in cells:
        nb = int(nbands(c)) if callable(nbands) else int(nbands)
        inp = sysm.kpoint_inputs(c, ecut, kfrac)
        kc = _context(dz, inp)
        kc.set_preconditioner(dz.PRECOND_TPA)
        kin = inp.basis.kinetic
        conv = kc.hermitian_eigen_decomp_iterative(kin, nb + 4, dz.Options(max_iter=400, tol=1e-10))
        for t in (t_list if t_list is not None else range(1, t_max + 1)):
            r = kc.hermitian_eigen_decomp_iterative(kin, nb, dz.Options(max_iter=t, tol=1e-14))
            psi = r.vectors
            hpsi = kc.apply_hamiltonian_batched(psi)
            res = hpsi - r.values[:, None] * psi
            bands = range(nb)
            if bands_per_t is not None and nb > bands_per_t:
                bands = sorted(rng.choice(nb, size=bands_per_t, replace=False).tolist())
            for b in bands:
                rn = float(np.linalg.norm(res[b]))
                if rn < 1e-7:
                    continue
                cl = np.nonzero(np.abs(conv.values - conv.values[b]) < cluster_tol)[0]
                Y = conv.vectors[cl]
                y = Y.T @ (Y.conj() @ psi[b])
                ny = float(np.linalg.norm(y))
                if ny < min_overlap:
                    continue
                y /= ny
                delta = y - psi.T @ (psi.conj() @ y)
                dn = float(np.vdot(delta, delta).real)
                if dn < 1e-24:
                    continue
                ekin = float(np.sum(kin * np.abs(psi[b]) ** 2))
                feats.append(_features(kin, ekin, np.abs(res[b]), rn / np.sqrt(len(kin)), t - 1))
                ccs.append(np.conj(res[b]) * delta)
                ws.append(np.abs(res[b]) ** 2)
                dns.append(dn)
                kins.append(kin)
                lams.append(float(r.values[b]))
                off.append(off[-1] + len(kin))
        kc.close()
    if len(off) == 1:
        raise RuntimeError("precond_samples: no band passed the overlap test")
    return {
        "off": np.array(off, dtype=np.int32),
        "feat": np.concatenate(feats).astype(np.float32),
        "cc": np.concatenate(ccs),
        "w": np.concatenate(ws),
        "dnorm": np.array(dns),
        "kin": np.concatenate(kins),
        "lam": np.array(lams),
    }


def fixed_loss(samples, kind: str) -> float:
    """The training loss of a fixed preconditioner on the same samples (host arithmetic)."""
    off = samples["off"]
    nb = len(off) - 1
    band = np.repeat(np.arange(nb), np.diff(off))
    kin = samples["kin"]
    if kind == "reference":
        den = kin - samples["lam"][band]
        den = np.where(np.abs(den) < 1e-8, np.where(den >= 0, 1e-8, -1e-8), den)
        m = 1.0 / den
    else:
        x = np.exp(samples["feat"][:, 0].astype(np.float64)) - 0.05
        num = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
        m = num / (num + 16.0 * x ** 4)
    cc, w = samples["cc"], samples["w"]
    A = np.bincount(band, weights=(m * cc).real, minlength=nb) + 1j * np.bincount(band, weights=(m * cc).imag, minlength=nb)
    Q = np.bincount(band, weights=m * m * w, minlength=nb)
    return float(np.mean(1.0 - np.abs(A) ** 2 / (Q * samples["dnorm"])))


def init_params(seed: int = 0, scale: float = 0.3) -> np.ndarray:
    """Initial weights (layout of DFTCUDA_PRECOND_MLP_PARAMS: W1, b1, W2, b2, w3, b3): random hidden
    layers and a zero output layer, so the untrained preconditioner is exactly Teter-Payne-Allan."""
    H = 64
    rng = np.random.default_rng(seed)
    parts = [
        rng.normal(0.0, scale, H * 3),
        rng.normal(0.0, scale, H),
        rng.normal(0.0, scale / np.sqrt(H), H * H),
        rng.normal(0.0, scale, H),
        np.zeros(H),
        [0.0],
    ]
    return np.concatenate(parts).astype(np.float32)


def train_precond(dz, samples, steps: int = 1500, lr: float = 2e-3, seed: int = 0):
    p0 = init_params(seed)
    p, hist = dz.precond_mlp_train(p0, samples["off"], samples["feat"], samples["cc"], samples["w"], samples["dnorm"], steps, lr)
    return p, hist


def scale_output(params, alpha: float) -> np.ndarray:
    """The network with its output layer (w3, b3) scaled by alpha: m = K_TPA exp(alpha z_theta).
    alpha = 0 is exactly Teter-Payne-Allan, alpha = 1 the trained network."""
    H = 64
    p = np.array(params, dtype=np.float32)
    o = 3 * H + H + H * H + H
    p[o:o + H + 1] *= np.float32(alpha)
    return p


def davidson_h_applies(dz, cells, ecut: float, nbands, kind, params=None, tol: float = 1e-6) -> float:
    """Mean H applications of the device Davidson solver (random start, to tol) over the cells."""
    n = []
    for c in cells:
        inp = sysm.kpoint_inputs(c, ecut, (0.0, 0.0, 0.0))
        nb = int(nbands(c)) if callable(nbands) else int(nbands)
        kc = _context(dz, inp)
        kc.set_preconditioner(kind, params)
        r = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, nb, dz.Options(max_iter=300, tol=tol))
        n.append(r.h_applies if r.converged else 10 * r.h_applies)
        kc.close()
    return float(np.mean(n))


def without_iteration_input(samples, params):
    """The network made independent of its iteration input: the feature zeroed in the samples and its
    column of W1 (W1[64][3], input 2) zeroed in the parameters, so it stays zero under training.
    The Davidson solves inside an SCF run restart the iteration count at 0 from warm vectors, a state
    that the random-start trajectories of the training data label as the earliest, roughest phase."""
    s = dict(samples)
    f = np.array(samples["feat"], dtype=np.float32, copy=True)
    f[:, 2] = 0.0
    s["feat"] = f
    p = np.array(params, dtype=np.float32, copy=True)
    p[2:3 * 64:3] = 0.0
    return s, p


def scf_h_applies(dz, cells, ecut: float, kind, params=None, extra_bands: int = 8) -> float:
    """Mean over the cells of the H applications that a resident FP64 SCF run needs (Gamma, occupied
    bands + extra_bands, the reference's mixing and eigensolver defaults, warm-started Davidson each
    step) to reach a density residual of 1e-6 with the given preconditioner; a run that does not
    converge in 60 steps counts three times.  This is the regime the preconditioner serves inside
    the SCF: every Davidson solve after the first starts from the previous step's vectors."""
    n = []
    for c in cells:
        nb = int(round(c.nelec / 2.0)) + extra_bands
        b = scfm.GpuBackend(dz, "fp64", precond=(kind, params), resident=True)
        r = scfm.run_scf(c, scfm.ScfParams(ecut=ecut, kmesh=(1, 1, 1), nbands=nb, convergence=1e-6, max_iter=60), b)
        b.close()
        cost = float(sum(s[2] for s in b.solves))
        n.append(cost if r.converged else 3.0 * cost)
    return float(np.mean(n))


def train_and_select(dz, samples, val_cells, ecut: float, nbands, steps: int, lr: float, chunks: int = 4,
                     alphas=(0.1, 0.25, 0.5, 1.0), iteration_input: bool = False, objective: str = "scf"):
    """The loss (1 - cos^2 against the projected correction) does not rank preconditioners by what
    the solver needs, so the model is selected on the solver itself: the network is trained in
    `chunks` segments of steps/chunks Adam steps, and every snapshot, with its output layer scaled by
    each alpha, is scored on the validation cells by the mean H applications of whole SCF runs
    (objective "scf", the default: warm-started solves, where a network that only shortens
    random-start solves was measured to lengthen the Si216 SCF from 14 to 35 steps) or of single
    random-start Davidson solves (objective "davidson").
    Returns (params of the best snapshot and scale, loss history, selection table); the table holds
    TPA (alpha = 0) for comparison, and the best entry can be TPA itself."""
    p = init_params(0)
    if not iteration_input:
        samples, p = without_iteration_input(samples, p)
    hist = []

    def cost(kind, q):
        if objective == "scf":
            return scf_h_applies(dz, val_cells, ecut, kind, q)
        return davidson_h_applies(dz, val_cells, ecut, nbands, kind, q)

    tpa = cost(dz.PRECOND_TPA, None)
    table = [{"steps": 0, "alpha": 0.0, "h_applies": tpa}]
    best = (tpa, scale_output(p, 0.0), 0, 0.0)
    per = max(1, steps // chunks)
    for k in range(chunks):
        p, h = dz.precond_mlp_train(p, samples["off"], samples["feat"], samples["cc"], samples["w"], samples["dnorm"], per, lr)
        hist.append(h)
        for a in alphas:
            q = scale_output(p, a)
            ha = cost(dz.PRECOND_MLP, q)
            table.append({"steps": per * (k + 1), "alpha": a, "h_applies": ha})
            if ha < best[0]:
                best = (ha, q, per * (k + 1), a)
    return best[1], np.concatenate(hist), {"objective": objective, "table": table,
                                           "chosen": {"steps": best[2], "alpha": best[3], "h_applies": best[0]},
                                           "tpa_h_applies": tpa}


def eval_loss(dz, params, samples) -> float:
    return dz.precond_mlp_loss_grad(params, samples["off"], samples["feat"], samples["cc"], samples["w"], samples["dnorm"])[0]


def evaluate_precond(dz, cells, ecut: float, nbands: int, params, tol: float = 1e-6, kfrac=(0.0, 0.0, 0.0)) -> dict:
    """Davidson iterations and H applications to reach tol from the random start, per preconditioner."""
    out = {"reference": [], "tpa": [], "mlp": []}
    for c in cells:
        inp = sysm.kpoint_inputs(c, ecut, kfrac)
        nb = int(nbands(c)) if callable(nbands) else int(nbands)
        for kind, key in ((dz.PRECOND_REFERENCE, "reference"), (dz.PRECOND_TPA, "tpa"), (dz.PRECOND_MLP, "mlp")):
            kc = _context(dz, inp)
            kc.set_preconditioner(kind, params if kind == dz.PRECOND_MLP else None)
            r = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, nb, dz.Options(max_iter=300, tol=tol))
            out[key].append({"iterations": r.iterations, "h_applies": r.h_applies, "converged": r.converged})
            kc.close()
    summ = {}
    for key, rs in out.items():
        summ[key] = {
            "mean_iterations": float(np.mean([r["iterations"] for r in rs])),
            "mean_h_applies": float(np.mean([r["h_applies"] for r in rs])),
            "all_converged": all(r["converged"] for r in rs),
        }
    return summ


def evaluate_si216(dz, params, tol: float = 1e-6, max_iter: int = 400) -> dict:
    """The learned preconditioner on the benchmark cell: one Davidson solve of the Si216 cell (3x3x3
    conventional, seed 3, 25 Ry, Gamma, 448 bands, the reference's defaults otherwise) from the
    random start to the same residual tol, per preconditioner: iterations, H applications and the
    solve's wall time (FP64 contexts, device-resident)."""
    import torch

    c = sysm.crystal("si216", 3)
    inp = sysm.kpoint_inputs(c, 25.0, (0.0, 0.0, 0.0))
    out = {}
    for kind, key in ((dz.PRECOND_REFERENCE, "reference"), (dz.PRECOND_TPA, "tpa"), (dz.PRECOND_MLP, "mlp")):
        kc = _context(dz, inp)
        kc.set_preconditioner(kind, params if kind == dz.PRECOND_MLP else None)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, 448, dz.Options(max_iter=max_iter, tol=tol))
        torch.cuda.synchronize()
        out[key] = {"iterations": r.iterations, "h_applies": r.h_applies, "wall_s": round(time.perf_counter() - t0, 3),
                    "converged": bool(r.converged), "max_residual": float(r.max_residual), "lowest_eigenvalue": float(r.values[0])}
        kc.close()
    return out


def load_precond_weights(path: str = PRECOND_WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        return np.asarray(z["params"], dtype=np.float32)


# ---- learned first density -------------------------------------------------------------------


def fno_input(c, ecut: float):
    """(dims, u [2][N] = atomic channels / mean density, rho_atomic [N], mean density)."""
    dims = sysm.fft_box(ecut, c.recip)
    ch = sysm.atomic_density_channels(c, dims)
    mean = c.nelec / c.volume
    return dims, ch / mean, ch.sum(axis=0), mean


def fno_initial_density(dz, params, c, ecut: float) -> np.ndarray:
    """rho0 = rho_atomic + mean * FNO(u), clipped at 1e-3 mean and renormalised to N_e."""
    dims, u, rho_at, mean = fno_input(c, ecut)
    d = dz.fno_forward(params, u, dims).astype(np.float64)
    rho = np.maximum(rho_at + mean * d, 1e-3 * mean)
    return rho * (c.nelec / (rho.mean() * c.volume))


def _scf_params(ecut, kmesh, nbands, tol, init=None, smearing=None, warmup_steps=2):
    return scfm.ScfParams(ecut=ecut, kmesh=kmesh, nbands=nbands, convergence=tol, max_iter=80, smearing=smearing, initial_density=init,
                          warmup_steps=warmup_steps)


FNO_SMEARING = 0.005  # Ry, Fermi-Dirac: random SiGe occupancies can close the gap of fixed occupations


def fno_samples(dz, cells, ecut: float, nbands: int, kmesh=(2, 2, 2), tol: float = 1e-7):
    """(dims, u, target) per cell; target = (rho_scf - rho_atomic) / mean from a plain SCF run."""
    out = []
    for c in cells:
        dims, u, rho_at, mean = fno_input(c, ecut)
        b = scfm.GpuBackend(dz, "fp64")
        r = scfm.run_scf(c, _scf_params(ecut, kmesh, nbands, tol, smearing=FNO_SMEARING), b)
        b.close()
        out.append((dims, u, (r.rho - rho_at) / mean))
    return out


def fno_init_params(seed: int = 0, spec_scale: float = 0.5, scale: float = 0.3) -> np.ndarray:
    """Random initial FNO weights (layout of DFTCUDA_FNO_PARAMS)."""
    W, K, L = 8, 16 ** 3, 4
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, scale, W * 2), np.zeros(W)]
    for _ in range(L):
        parts.append(rng.normal(0.0, spec_scale / W, 2 * K * W * W))
        parts.append(rng.normal(0.0, scale / np.sqrt(W), W * W))
        parts.append(np.zeros(W))
    parts.append(rng.normal(0.0, scale / np.sqrt(W), W))
    parts.append([0.0])
    return np.concatenate(parts).astype(np.float32)


def evaluate_fno(dz, params, cells, ecut: float, nbands: int, kmesh=(2, 2, 2), tol: float = 1e-6) -> dict:
    """SCF iterations from the flat start (the reference default), the atomic superposition and the
    learned start; plus the initial density error against the converged density."""
    rows = []
    for c in cells:
        dims, u, rho_at, mean = fno_input(c, ecut)
        rho_fno = fno_initial_density(dz, params, c, ecut)
        starts = {"flat": None, "atomic": rho_at * (c.nelec / (rho_at.mean() * c.volume)), "fno": rho_fno, "fno_no_warmup": rho_fno}
        row = {}
        conv_rho = None
        for name, init in starts.items():
            b = scfm.GpuBackend(dz, "fp64")
            # the reference's loose-tolerance warm-up iterations (density.zig:128-183) exist for poor
            # starting densities; the learned start is also run without them
            wu = 0 if name == "fno_no_warmup" else 2
            r = scfm.run_scf(c, _scf_params(ecut, kmesh, nbands, tol, init, smearing=FNO_SMEARING, warmup_steps=wu), b)
            b.close()
            row[name] = {"iterations": r.iterations, "converged": r.converged, "energy_per_atom": r.energy_per_atom, "wall_s": r.wall_s}
            if name == "flat":
                conv_rho = r.rho
        for name, init in starts.items():
            if init is not None:
                row[name]["initial_rms_error"] = float(np.sqrt(np.mean((init - conv_rho) ** 2)) / mean)
        rows.append(row)
    summ = {}
    for name in ("flat", "atomic", "fno", "fno_no_warmup"):
        summ[name] = {
            "mean_iterations": float(np.mean([r[name]["iterations"] for r in rows])),
            "all_converged": all(r[name]["converged"] for r in rows),
            "mean_wall_s": float(np.mean([r[name]["wall_s"] for r in rows])),
        }
        if name != "flat":
            summ[name]["mean_initial_rms_error"] = float(np.mean([r[name]["initial_rms_error"] for r in rows]))
    summ["max_energy_spread_per_atom"] = float(max(max(r[n]["energy_per_atom"] for n in r) - min(r[n]["energy_per_atom"] for n in r) for r in rows))
    return summ


def load_fno_weights(path: str = FNO_WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        return np.asarray(z["params"], dtype=np.float32)


def main(argv=None):
    import importlib

    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=("precond", "fno", "precond-eval"))
    ap.add_argument("--cells", choices=("sitrain", "si8d"), default="sitrain",
                    help="sitrain: 200 seeded Si cells of 8-64 atoms (seeds 1000..), si8d: strained Si8 cells")
    ap.add_argument("--train-cells", type=int, default=200)
    ap.add_argument("--eval-cells", type=int, default=16)
    ap.add_argument("--ecut", type=float, default=25.0,
                    help="cutoff (Ry) of the training data, the selection runs and the held-out solves: the "
                         "Si216 benchmark's, so that |k+G|^2 / E_kin spans the same range")
    ap.add_argument("--nbands", type=int, default=16)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=PRECOND_WEIGHTS)
    ap.add_argument("--fno-train-cells", type=int, default=64)
    ap.add_argument("--fno-eval-cells", type=int, default=8)
    ap.add_argument("--fno-steps", type=int, default=400)
    ap.add_argument("--fno-lr", type=float, default=2e-3)
    ap.add_argument("--eval-only", action="store_true", help="fno: evaluate the shipped weights, no training")
    a = ap.parse_args(argv)
    dz = importlib.import_module(__package__)
    if a.what == "fno":
        return main_fno(dz, a)
    if a.what == "precond-eval":
        print(json.dumps({"si216": evaluate_si216(dz, load_precond_weights(a.out))}), flush=True)
        return
    t0 = time.perf_counter()
    if a.cells == "sitrain":
        # the occupied bands of each cell; a few Davidson iterations of each trajectory and at most
        # 12 bands of each iteration keep the 200 cells' data under ~1 GB
        train_cells = [sysm.crystal("sitrain", 1000 + i) for i in range(a.train_cells)]
        eval_cells = [sysm.crystal("sitrain", 1200 + i) for i in range(a.eval_cells)]
        nb = lambda c: int(round(c.nelec / 2.0))
        kw = dict(t_list=(1, 2, 4, 7, 11, 16), bands_per_t=12)
        tr = precond_samples(dz, train_cells, a.ecut, nb, seed=1, **kw)
        ev = precond_samples(dz, eval_cells, a.ecut, nb, seed=2, **kw)
        # selection by a whole SCF run on a 144-atom validation cell (3 x 3 x 2, the family's recipe;
        # SCF runs of 48-64-atom cells did not rank the networks as the 216-atom SCF does), the
        # Davidson comparison on the held-out cells of the training family
        first = eval_cells[: min(6, len(eval_cells))]
        val_cells = [sysm.crystal("sival", 5000)]
        dav_cells, dav_nb = eval_cells[len(first):] or first, nb
    else:
        train_cells = [sysm.crystal("si8d", 1000 + i) for i in range(a.train_cells)]
        eval_cells = [sysm.crystal("si8d", 1200 + i) for i in range(a.eval_cells)]
        tr = precond_samples(dz, train_cells, a.ecut, a.nbands)
        ev = precond_samples(dz, eval_cells, a.ecut, a.nbands)
        dav_cells, dav_nb = eval_cells, a.nbands
    t1 = time.perf_counter()
    selection = None
    if a.cells == "sitrain":
        p, hist, selection = train_and_select(dz, tr, val_cells, a.ecut, nb, a.steps, a.lr)
    else:
        p, hist = train_precond(dz, tr, a.steps, a.lr)
    t2 = time.perf_counter()
    report = {
        "cells": a.cells,
        "train_cells": len(train_cells),
        "train_atoms": sorted({len(c.atom_species) for c in train_cells}),
        "train_bands": int(len(tr["off"]) - 1),
        "train_plane_waves": int(tr["feat"].shape[0]),
        "data_seconds": round(t1 - t0, 2),
        "train_seconds": round(t2 - t1, 2),
        "loss_first": float(hist[0]),
        "loss_last": float(hist[-1]),
        "heldout_loss": eval_loss(dz, p, ev),
        "heldout_loss_initial_weights_tpa": eval_loss(dz, init_params(0), ev),
        "heldout_loss_reference_diagonal": fixed_loss(ev, "reference"),
        "heldout_loss_tpa": fixed_loss(ev, "tpa"),
        "heldout_davidson": evaluate_precond(dz, dav_cells, a.ecut, dav_nb, p),
    }
    if selection is not None:
        report["selection"] = selection
    if a.cells == "sitrain":
        report["si216"] = evaluate_si216(dz, p)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.savez(a.out, params=p, loss_history=hist.astype(np.float32), report=json.dumps(report))
    print(json.dumps(report), flush=True)


def main_fno(dz, a):
    """SiGe8 cells (20 Ry, 2x2x2 k, 20 bands): train on seeds 2000.., evaluate on seeds 2400.."""
    ecut, nb = 20.0, 20
    if a.eval_only:
        p = load_fno_weights()
        cells = [sysm.crystal("sige8", 2400 + i) for i in range(a.fno_eval_cells)]
        print(json.dumps({"heldout_scf": evaluate_fno(dz, p, cells, ecut, nb)}), flush=True)
        return
    t0 = time.perf_counter()
    train = fno_samples(dz, [sysm.crystal("sige8", 2000 + i) for i in range(a.fno_train_cells)], ecut, nb)
    heldout_cells = [sysm.crystal("sige8", 2400 + i) for i in range(a.fno_eval_cells)]
    heldout = fno_samples(dz, heldout_cells, ecut, nb)
    t1 = time.perf_counter()
    p0 = fno_init_params(0)
    p, hist = dz.fno_train(p0, train, a.fno_steps, a.fno_lr)
    t2 = time.perf_counter()
    zero = np.zeros_like(p0)
    report = {
        "train_cells": len(train),
        "data_seconds": round(t1 - t0, 2),
        "train_seconds": round(t2 - t1, 2),
        "loss_first": float(hist[0]),
        "loss_last": float(hist[-1]),
        "heldout_loss": dz.fno_loss_grad(p, heldout)[0],
        "heldout_loss_atomic_start": dz.fno_loss_grad(zero, heldout)[0],
        "heldout_scf": evaluate_fno(dz, p, heldout_cells, ecut, nb),
    }
    out = a.out if a.out != PRECOND_WEIGHTS else FNO_WEIGHTS
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.savez(out, params=p, loss_history=hist.astype(np.float32), report=json.dumps(report))
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
