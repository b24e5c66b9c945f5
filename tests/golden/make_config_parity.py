"""Oracle results at the benchmark configurations' own sizes, for the GPU parity tests.

The oracle (numpy restatement of the reference) is too slow to rerun inside every GPU test at these
sizes, so its results are computed once by this script and committed as config_parity.json:

  si64_gamma_davidson  Si64 (2x2x2 conventional, seed 1, N(0, 0.02 A) displacements), 30 Ry, Gamma,
                       160 bands: the oracle's serial Davidson (lobpcg/serial.zig:55-307) from the
                       reference's LCG start with max_subspace 648, tol 1e-6.  Eigenvalues (Ry).
  si2_444_scf          Si2 (config 1): LDA-PZ, 20 Ry, 4x4x4 unshifted MP mesh (k and -k folded:
                       36 points), 8 bands, fixed occupations, Pulay 8 / beta 0.3, tight eigensolver
                       (1e-10), no warm-up, SCF to 1e-10.  Energy per atom and every eigenvalue.
  al4_888_three_k      Al4 (config 3: conventional FCC, seed 2 strain), LDA-PZ, 25 Ry, three points of
                       the 8x8x8 mesh with different plane-wave counts (equal weights), 12 bands,
                       Fermi-Dirac 0.02 Ry.  Energy per atom and every eigenvalue.

Run from the repository root:  python tests/golden/make_config_parity.py [name ...]
"""
from __future__ import annotations

import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
OUT = os.path.join(HERE, "config_parity.json")

SI2_PARAMS = dict(ecut=20.0, kmesh=(4, 4, 4), nbands=8, convergence=1e-10, iterative_max_iter=300, iterative_tol=1e-10,
                  warmup_steps=0, max_iter=60)
AL4_KPOINTS = [((0.0, 0.0, 0.0), 1.0 / 3.0), ((0.125, 0.0, 0.0), 1.0 / 3.0), ((0.375, 0.25, 0.125), 1.0 / 3.0)]
AL4_PARAMS = dict(ecut=25.0, kmesh=(8, 8, 8), nbands=12, convergence=1e-10, iterative_max_iter=300, iterative_tol=1e-10,
                  warmup_steps=0, max_iter=60, smearing=0.02)
SI64_OPTS = dict(max_iter=200, tol=1e-6, max_subspace=648)


def si64_gamma_davidson():
    from oracle import cases, lobpcg

    kp = cases.make_kproblem(cases.make_cell("si64", 1), 30.0)
    ctx = kp.ctx
    t = time.time()
    r = lobpcg.solve(lobpcg.Operator(ctx.n, ctx.apply_batch), ctx.basis.kinetic, 160, lobpcg.Options(**SI64_OPTS))
    return dict(n_pw=int(ctx.n), dims=[kp.grid.nx, kp.grid.ny, kp.grid.nz], nbands=160, opts=SI64_OPTS,
                eigenvalues=[float(v) for v in r.values], iterations=int(getattr(r, "iterations", -1)),
                oracle_seconds=round(time.time() - t, 1))


def _scf(cell_name, seed, params):
    import dftzig_loader
    from tests.helpers import OracleBackend

    dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal(cell_name, seed)
    t = time.time()
    r = scf.run_scf(c, scf.ScfParams(**params), OracleBackend())
    return dict(converged=bool(r.converged), iterations=int(r.iterations), energy_per_atom=float(r.energy_per_atom),
                eigenvalues=[[float(v) for v in np.asarray(e)] for e in r.eigenvalues], oracle_seconds=round(time.time() - t, 1))


def si2_444_scf():
    d = _scf("si2", 1, SI2_PARAMS)
    d["params"] = {k: (list(v) if isinstance(v, tuple) else v) for k, v in SI2_PARAMS.items()}
    return d


def al4_888_three_k():
    p = dict(AL4_PARAMS, kpoints=AL4_KPOINTS)
    d = _scf("al4", 2, p)
    d["params"] = {k: (list(v) if isinstance(v, tuple) else v) for k, v in AL4_PARAMS.items()}
    d["kpoints"] = [[list(k), w] for k, w in AL4_KPOINTS]
    return d


CASES = {"si64_gamma_davidson": si64_gamma_davidson, "si2_444_scf": si2_444_scf, "al4_888_three_k": al4_888_three_k}


def main(names):
    for name in names or list(CASES):
        t = time.time()
        res = CASES[name]()
        print(f"{name}: {time.time() - t:.1f} s", flush=True)
        out = json.load(open(OUT)) if os.path.exists(OUT) else {}  # re-read: cases may run in parallel
        out[name] = res
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
