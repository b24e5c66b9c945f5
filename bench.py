#!/usr/bin/env python
"""H|psi> throughput and time-to-SCF of the dft-zig plane-wave hot path on B200.

Workload (one "step", default): one Davidson block of H|psi> (nbands + 4 = 452 columns) at the Gamma
point of the Si216 cell -- 3x3x3 conventional Si supercell with seeded N(0, 0.05 A) displacements
(seed 3), 25 Ry cutoff, 108^3 FFT box, 61,565 plane waves, 216 atoms of Kleinman-Bylander
projectors, FP64.  --cell si64 selects the Si64 block instead (2x2x2 supercell, 30 Ry, 75^3 box,
2x2x2 Monkhorst-Pack mesh, 8 k-points x 164 columns).  Synthetic inputs: seeded wavefunction
coefficients; the species are synthetic GTH-form pseudopotentials (the reference ships none).

  value        algorithmic HBM GB/s of the device-resident operator: columns x B_alg / device time,
               B_alg = 2 n_pw s + 2 N s + 8 N / nb per column (s = 16 B; the shared-memory-resident
               P = 1 form of the per-band byte count), inputs resident in HBM; the 890 MB of inputs
               and outputs per step exceed the 126 MB L2, so no flush is needed.
  e2e          the same metric through the C ABI (dftcuda_apply_h_batch) from pinned host buffers:
               host->device copy of every column and device->host copy of every result inside the timing.
  time_to_scf  (Si216, one GPU) wall seconds until |E - E_target| < 1e-6 Ry/atom, plain FP64 against
               learned + mixed precision, E_target the energy of the plain FP64 run carried on to a
               density residual of 1e-8 (its own time-to-SCF is the wall time of its first iteration
               within the bar), with the clocks sampled during both runs.

--impl reference times the CPU restatement of the reference's path (the oracle: numpy FFT + BLAS)
on the same workload, a bounded column sample spread over all host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# H|psi> workloads: cell, seed, cutoff (Ry), k-mesh, bands; the Davidson block is nbands + 4 columns
# (lobpcg/serial.zig:78-82)
WORKLOADS = {
    "si216": dict(cell="si216", seed=3, ecut=25.0, kmesh=(1, 1, 1), nbands=448,
                  label="Si216 3x3x3 conventional, 25 Ry, 108^3 box, Gamma, 452-column Davidson block, FP64 H|psi>"),
    "si64": dict(cell="si64", seed=1, ecut=30.0, kmesh=(2, 2, 2), nbands=160,
                 label="Si64 2x2x2 conventional, 30 Ry, 75^3 box, 2x2x2 MP (8 k), 164-column Davidson block, FP64 H|psi>"),
}
CELL, SEED, ECUT, KMESH, NBANDS = "si64", 1, 30.0, (2, 2, 2), 160  # the Si64 cell of the profiling cases
S = 16  # bytes per FP64 complex
# The three local passes of each layout (the library's profile reports which ran: 0 generic, 1 plane
# layout, 2 stick layout).
LOCAL_KERNELS = {0: ("k_plane_inv", "k_xline", "k_plane_fwd"), 1: ("k_plane_inv5", "k_xline5", "k_plane_fwd5"),
                 2: ("k_stick_inv", "k_zplane", "k_stick_fwd")}
# Measured DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum) of the three local passes
# per column, FP64, keyed by (cell, layout): from one application of a small Gamma case of the cell
# (Si64: 32 columns, Si216: 16 columns), scaled to a block by the columns processed.
LOCAL_DRAM_BYTES_PER_COLUMN = {("si64", 1): 315.0e6 / 32, ("si216", 2): 149.0e6 / 16}
DRAM_SOURCE = {("si64", 1): "profiles/local_kernels_dram_traffic_si64_fp64.md",
               ("si216", 2): "profiles/local_kernels_dram_traffic_si216_sticks_fp64.md"}


# Complex GEMM shapes of the Si216 Davidson step (n_pw = 61,565, 448 bands, subspace up to 1,800):
# M, N, K, conj_a, description.  out(r, c) = sum_k op(A(r, k)) B(c, k), A and B row-major [rows][K].
GEMM_SHAPES = {
    "gram1344": (1344, 1344, 120000, True, "Gram V^H W, 1344 x 1344, K = 120,000"),
    "t448x1344": (1344, 448, 61565, True, "new Rayleigh-Ritz columns V^H W_new, 1344 x 448, K = n_pw"),
    "rot448": (61565, 448, 1344, False, "Ritz rotation V C, n_pw x 448, K = 1344"),
    "proj864": (864, 452, 61565, True, "projections <beta|psi>, 864 projectors x 452 columns, K = n_pw"),
}


def run_gemm_workload(args):
    """The library's complex GEMM (dftcuda_complex_gemm) on the Si216 Davidson shapes: seeded
    complex128 operands resident on the device, one warm-up call, then the fastest of three calls
    (host clock around the synchronous call: kernels plus one stream sync, no allocation after the
    first call).  Error = max |out - out_FP64| / max |out_FP64|."""
    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    prec_of = {"fp64": dz.PRECISION_FP64, "tf32x3": dz.PRECISION_TF32X3, "tf32": dz.PRECISION_TF32}
    gen = torch.Generator(device="cuda").manual_seed(0)
    out = {}
    for name in [s for s in args.gemm_shapes.split(",") if s]:
        M, N, K, conj_a, desc = GEMM_SHAPES[name]
        a = torch.randn(M, K, dtype=torch.complex128, device="cuda", generator=gen)
        b = torch.randn(N, K, dtype=torch.complex128, device="cuda", generator=gen)
        o = torch.zeros(N, M, dtype=torch.complex128, device="cuda").T
        ref = torch.zeros_like(o)
        dz.complex_gemm(a, b, ref, conj_a=conj_a, precision=dz.PRECISION_FP64)
        row = {"shape": desc}
        for pn in [p for p in args.gemm_precisions.split(",") if p]:
            dz.complex_gemm(a, b, o, conj_a=conj_a, precision=prec_of[pn])
            torch.cuda.synchronize()
            ts = []
            for _ in range(3):
                t0 = time.perf_counter()
                dz.complex_gemm(a, b, o, conj_a=conj_a, precision=prec_of[pn])
                ts.append(time.perf_counter() - t0)
            err = float((o - ref).abs().max() / ref.abs().max())
            row[pn] = {"ms": round(1e3 * min(ts), 3), "useful_tflops": round(8.0 * M * N * K / min(ts) / 1e12, 1), "rel_err": err}
        out[name] = row
        del a, b, o, ref
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "complex GEMM, Si216 Davidson shapes", "useful_flops": "8 M N K", "shapes": out}), flush=True)


def bytes_per_column(npw: int, N: int, nb: int) -> float:
    return 2.0 * npw * S + 2.0 * N * S + 8.0 * N / nb


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cell", choices=tuple(WORKLOADS), default="si216", help="cell of the H|psi> workload")
    ap.add_argument("--no-scf", action="store_true", help="skip the Si216 time-to-SCF object of the default line")
    ap.add_argument("--no-variants", action="store_true", help="skip the FP32 / TF32 variants of the H|psi> step")
    ap.add_argument("--autotune", action="store_true",
                    help="run the context autotuner (layout, workspace budget, projector split-K) before timing")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--profile-case", action="store_true", help="small single-k case for ncu captures: Gamma, 32 columns, 2 applications")
    ap.add_argument("--workload", choices=("hpsi", "scf", "scf64", "scf216", "al4", "cells", "eig", "heev", "gemm", "potential"),
                    default="hpsi",
                    help="hpsi: H|psi> GB/s (default); scf: time-to-SCF Si2; scf64: time-to-SCF Si64, mixed vs FP64; "
                         "scf216: time-to-SCF Si216 (Gamma, 448 bands), FP64 vs learned+mixed; "
                         "al4: time-to-SCF Al4 8x8x8 (260 k-points, batched), FP64 vs mixed; "
                         "cells: many-cell SiGe8 SCF throughput, atomic vs learned start; "
                         "eig: one Si64 Gamma Davidson solve (profiling case); "
                         "heev: the subspace eigensolver on a seeded Hermitian matrix (--heev-m, lowest m/3 pairs); "
                         "gemm: the library's complex GEMM on the Si216 Davidson shapes (--gemm-shapes), FP64 / 3xTF32 / TF32; "
                         "potential: the Si216 box's potential build, Pulay step and standalone 3D FFTs")
    ap.add_argument("--eig-precond", choices=("reference", "tpa", "mlp"), default="reference",
                    help="preconditioner of --workload eig (mlp: the shipped trained weights)")
    ap.add_argument("--gemm-shapes", default="gram1344,t448x1344,rot448,proj864",
                    help="comma list of --workload gemm shapes: " + ", ".join(f"{k} ({v[4]})" for k, v in GEMM_SHAPES.items()))
    ap.add_argument("--gemm-precisions", default="fp64,tf32x3,tf32", help="comma list of --workload gemm precisions")
    ap.add_argument("--heev-m", type=int, default=1344, help="matrix size of --workload heev")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="scf216: instead of time-to-SCF, run N SCF steps of each arm and print its kernel-time "
                         "table (CUPTI activity records through torch.profiler)")
    ap.add_argument("--eig-iters", type=int, default=6, help="Davidson iterations of --workload eig")
    ap.add_argument("--eig-tol", type=float, default=1e-9, help="residual tolerance of --workload eig")
    ap.add_argument("--eig-cell", choices=("si64", "si216"), default="si64", help="cell of --workload eig")
    ap.add_argument("--cells", type=int, default=16, help="cells of the many-cell workload")
    ap.add_argument("--cells-starts", default="atomic,fno", help="starting densities of the many-cell workload (comma list)")
    ap.add_argument("--xc", choices=("lda", "pbe"), default="pbe", help="functional of the Si64 time-to-SCF workload")
    ap.add_argument("--switch-drho", type=float, default=1.5e-5,
                    help="density residual at which the Si216 learned+mixed run switches to FP64 (its TF32X3 "
                         "residuals track the FP64 run's to 1e-5; the stall rule still switches earlier on a floor)")
    ap.add_argument("--precision", choices=("fp64", "fp32", "tf32"), default="fp64",
                    help="context precision of --profile-case (tf32 = TF32 GEMMs) and --workload eig (tf32 = TF32X3)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f,
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [v.strip() for v in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax.append(float(p[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_inputs(w):
    import dftzig_loader

    dz = dftzig_loader.load()
    import importlib

    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal(w["cell"], w["seed"])
    kpts = system.monkhorst_pack(w["kmesh"])
    dims = system.fft_box(w["ecut"], c.recip)
    tables = [[system.radial_table(sp, i, w["ecut"]) for i in range(len(sp.betas))] for sp in c.species]
    vloc = system.local_potential(c, dims, w["ecut"])
    ins = [system.kpoint_inputs(c, w["ecut"], k, dims=dims, local_r=vloc, tables=tables) for k, _ in kpts]
    return dz, c, kpts, dims, ins


def run_ours(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    w = WORKLOADS[args.cell]
    NCOLS = w["nbands"] + 4
    dz, c, kpts, dims, ins = workload_inputs(w)
    N = dims[0] * dims[1] * dims[2]
    ctxs = []
    for inp in ins:
        kc = dz.KpointContext(dims[0], dims[1], dims[2], inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart)
        kc.set_vloc(inp.local_r)
        kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
        ctxs.append(kc)
    tuned = [kc.autotune(NCOLS) for kc in ctxs] if args.autotune else None
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    xs, ys = [], []
    for kc in ctxs:
        x = torch.randn((NCOLS, kc.n), dtype=torch.complex128, device="cuda", generator=gen)
        xs.append(x)
        ys.append(torch.empty_like(x))
    # A dedicated stream: the legacy default stream's handle is 0, which the C ABI reads as
    # "use the context's own stream".
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def step():
        for kc, x, y in zip(ctxs, xs, ys):
            kc.apply_hamiltonian_async(x, y, NCOLS, sptr)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    cols_per_step = NCOLS * len(ctxs)
    algo_bytes_step = sum(NCOLS * bytes_per_column(kc.n, N, NCOLS) for kc in ctxs)

    sampler = ClockSampler(local)
    for kc in ctxs:
        kc.set_profiling(True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    profs = [kc.profile() for kc in ctxs]
    for kc in ctxs:
        kc.set_profiling(False)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    # e2e through the C ABI from pinned host memory
    hx = [torch.from_numpy(x.cpu().numpy()).pin_memory() for x in xs]
    hy = [torch.empty_like(h).pin_memory() for h in hx]

    def e2e_step():
        for kc, x, y in zip(ctxs, hx, hy):
            kc.apply_hamiltonian_batched(x, y, kc.n, NCOLS)

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    # check one column against the device-resident result
    ok = bool(np.allclose(hy[0].numpy()[:2], ys[0][:2].cpu().numpy(), rtol=1e-12, atol=1e-12))

    # roofline: the fused local operator (three passes) is the dominant work
    tot = {k: sum(p[k] for p in profs) for k in profs[0]}
    layout = int(profs[0]["local_layout"])
    local_kernels = LOCAL_KERNELS[layout]
    launches = int(tot["kernel_launches"])
    local_ns = tot["apply_local_ns"]
    npw_avg = float(np.mean([kc.n for kc in ctxs]))
    local_bytes = cols_per_step * args.steps * (2.0 * npw_avg * S + 2.0 * N * S + 8.0 * N / NCOLS)
    peak, peak_kind = load_peaks()
    achieved = local_bytes / (local_ns * 1e-9) / 1e9 if local_ns else None
    value = world * algo_bytes_step / (ms * 1e-3) / 1e9
    e2e_value = world * algo_bytes_step / (e2e_ms * 1e-3) / 1e9
    h2d = sum(x.numel() * 16 for x in hx)
    names = dict(zip(("local_plane_inv_ns", "local_xline_ns", "local_plane_fwd_ns"), local_kernels))
    names.update(nl_project_ns="projection GEMM", nl_dij_ns="D_ij", nl_backproject_ns="back-projection GEMM")
    kern = {
        k: {"kernel": names[k], "ms_per_step": tot[k] / 1e6 / args.steps, "share": tot[k] / max(tot["apply_h_ns"], 1)}
        for k in ("local_plane_inv_ns", "local_xline_ns", "local_plane_fwd_ns", "nl_project_ns", "nl_dij_ns", "nl_backproject_ns")
    }
    # The same workload with the FP32 FFT passes (FP64 projector GEMMs) and in TF32 mode (FP32 FFT
    # passes + tcgen05 TF32 projector GEMMs): device time per step, the same algorithmic byte count.
    variants = {}
    for label, prec in (() if args.no_variants else (("fp32_fft", dz.PRECISION_FP32), ("tf32", dz.PRECISION_TF32))):
        vctx = []
        for inp in ins:
            kc = dz.KpointContext(dims[0], dims[1], dims[2], inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, prec)
            kc.set_vloc(inp.local_r)
            kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
            vctx.append(kc)
        for _ in range(3):
            for kc, x, y in zip(vctx, xs, ys):
                kc.apply_hamiltonian_async(x, y, NCOLS, sptr)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            for kc, x, y in zip(vctx, xs, ys):
                kc.apply_hamiltonian_async(x, y, NCOLS, sptr)
        f1.record(stream)
        torch.cuda.synchronize()
        vms = f0.elapsed_time(f1) / args.steps
        variants[label] = {"ms_per_step": round(vms, 3), "value": round(world * algo_bytes_step / (vms * 1e-3) / 1e9, 1), "unit": "GB/s"}
        for kc in vctx:
            kc.close()

    dram = LOCAL_DRAM_BYTES_PER_COLUMN.get((args.cell, layout))
    line = {
        "metric": "H|psi> HBM GB/s (algorithmic)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded wavefunctions; synthetic GTH-form Si pseudopotential)",
        "config": {
            "workload": w["label"],
            "columns_per_step": cols_per_step,
            "n_pw_mean": round(npw_avg, 1),
            "fft_box": list(dims),
            "bytes_per_column_alg": round(bytes_per_column(int(npw_avg), N, NCOLS)),
            "l2": f"inputs+outputs per step {2 * 16 * cols_per_step * npw_avg / 1e9:.2f} GB > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas x{world}",
        },
        "clocks": clocks,
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d, "timer": "host wall clock around synchronous C-ABI calls", "matches_device_result": ok},
        "gpu_launches": launches,
        "roofline": {
            "kernel": f"local H|psi>: {' + '.join(local_kernels)} (one {NCOLS}-column block)",
            "bound": "hbm",
            "achieved": round(achieved, 1) if achieved else None,
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None,
            "peak_source": peak_kind,
            # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the three passes per column,
            # from one ncu capture of a small Gamma case of the same cell, scaled to one block
            "traffic": round(dram * NCOLS) if dram else None,
            "traffic_source": DRAM_SOURCE.get((args.cell, layout)) if dram else None,
            "algorithmic_bytes": round(bytes_per_column(int(npw_avg), N, NCOLS) * NCOLS),
            "per": f"one {NCOLS}-column application of the local operator at one k-point",
        },
        "kernels": kern,
        "autotune": tuned,
        "variants": variants,
    }
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(w)
    if rank == 0 and world == 1 and args.cell == "si216" and not args.no_scf:
        for kc in ctxs:
            kc.close()
        ctxs = []
        del xs, ys, hx, hy
        torch.cuda.set_stream(torch.cuda.default_stream())  # the driver's torch work on the default stream
        torch.cuda.empty_cache()
        line["time_to_scf"] = time_to_scf_si216(dz, args, local)
    if world > 1:
        dist.destroy_process_group()
    for kc in ctxs:
        kc.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# CPU: the oracle (test infrastructure) timed as the reported baseline
# ---------------------------------------------------------------------------------------------


_CPU_PROBLEMS = {}


def _cpu_init(cell, seed, ecut, kfracs):
    """Pool initializer: one single-threaded process per core builds the oracle problem of every
    k-point once, so the timed steps contain H|psi> only."""
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from oracle import cases

    c = cases.make_cell(cell, seed)
    for i, kf in enumerate(kfracs):
        _CPU_PROBLEMS[i] = cases.make_kproblem(c, ecut, kf)


def _cpu_worker(task):
    import numpy as _np

    ki, ncols, seed = task
    kp = _CPU_PROBLEMS[ki]
    rng = _np.random.default_rng(seed)
    x = rng.normal(size=(ncols, kp.ctx.n)) + 1j * rng.normal(size=(ncols, kp.ctx.n))
    t0 = time.perf_counter()
    kp.ctx.apply_batch(x)
    dt = time.perf_counter() - t0
    return dt, ncols, kp.ctx.n, kp.grid.count


def cpu_baseline(w, cols: int = 0):
    """Single core: the oracle H|psi> on a column sample of the workload's first k-point (Gamma)."""
    import multiprocessing as mp

    cols = cols or (24 if w["cell"] == "si216" else 160)
    nb = w["nbands"] + 4
    ctx = mp.get_context("spawn")
    with ctx.Pool(1, initializer=_cpu_init, initargs=(w["cell"], w["seed"], w["ecut"], [(0.0, 0.0, 0.0)])) as pool:
        dt, nc, npw, N = pool.map(_cpu_worker, [(0, cols, 0)])[0]
    v = nc * bytes_per_column(npw, N, nb) / dt / 1e9
    return {"value": round(v, 4), "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": f"{nc} of the {nb} columns of H|psi> at Gamma, numpy oracle, one core, {dt:.1f} s"}


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle import cases

    w = WORKLOADS[args.cell]
    NCOLS = w["nbands"] + 4
    kpts = cases.monkhorst_pack(w["kmesh"])
    kfr = [tuple(float(v) for v in k) for k, _ in kpts]
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    # a bounded sample of the block per step: one column per process (Si216, one k-point), or 8
    # columns at each k-point (Si64)
    if len(kfr) == 1:
        tasks = [(0, 1, i) for i in range(cores)]
        sample_txt = f"{cores} of the {NCOLS} columns at Gamma per step, one per process"
    else:
        tasks = [(i, 8, i) for i in range(len(kfr))]
        sample_txt = f"8 of {NCOLS} columns at each of {len(kfr)} k-points per step"
    steps = max(1, args.steps)
    with ctx.Pool(cores, initializer=_cpu_init, initargs=(w["cell"], w["seed"], w["ecut"], kfr)) as pool:
        for _ in range(max(1, min(args.warmup, 1))):
            pool.map(_cpu_worker, tasks, chunksize=1)
        times = []
        done_bytes = 0.0
        for s in range(steps):
            t0 = time.perf_counter()
            res = pool.map(_cpu_worker, tasks, chunksize=1)
            dt = time.perf_counter() - t0
            times.append(dt)
            done_bytes += sum(nc * bytes_per_column(npw, N, NCOLS) for _, nc, npw, N in res)
    total_t = sum(times)
    v = done_bytes / total_t / 1e9
    sample = f"{sample_txt}, {cores} processes (numpy oracle; the reference binary needs Zig/FFTW/OpenBLAS, absent here)"
    line = {
        "impl": "reference",
        "metric": "H|psi> HBM GB/s (algorithmic)",
        "value": round(v, 4),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_t / steps * 1e3, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": w["label"], "sample": sample_txt},
        "cpu_baseline": {"value": round(v, 4), "unit": "GB/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def time_to_scf_si216(dz, args, device_index: int):
    """The headline comparison on Si216 (3x3x3 conventional, seed 3, 25 Ry, Gamma, 448 bands, LDA-PZ,
    fixed occupations, Pulay 8 / beta 0.3, the reference's eigensolver defaults, resident driver).
    Plain FP64 (reference preconditioner) runs on to a density residual of 1e-8; its final energy is
    the target, and its time-to-SCF is the wall time (setup included, from the start of the run) of
    its first iteration within 1e-6 Ry/atom of the target.  Learned + mixed precision (TF32X3 contexts
    with the trained MLP preconditioner, FP64 after the switch) then runs until it is within the same
    bar of the same target.  Clocks are sampled during both runs."""
    import importlib

    import torch

    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    learn = importlib.import_module("dftzig_b200.learn")
    c = system.crystal("si216", 3)
    natom = len(c.atom_species)
    base = dict(ecut=25.0, kmesh=(1, 1, 1), nbands=448, mixing_beta=0.3, pulay_history=8, max_iter=60)
    sampler = ClockSampler(device_index)
    sampler.start()
    torch.cuda.synchronize()
    b = scf.GpuBackend(dz, "fp64", resident=True)
    ref = scf.run_scf(c, scf.ScfParams(**base, convergence=1e-8), b)
    torch.cuda.synchronize()
    b.close()
    if not ref.converged:
        raise RuntimeError("the plain FP64 Si216 run did not converge")
    hit = next(h for h in ref.history if abs(h[1] - ref.energy) / natom < 1e-6)
    mlp = (dz.PRECOND_MLP, learn.load_precond_weights())
    p = scf.ScfParams(**base, convergence=1e-12, energy_target=ref.energy, energy_tol_per_atom=1e-6)
    b = scf.GpuBackend(dz, "mixed", precond=mlp, resident=True, switch_drho=args.switch_drho)
    r = scf.run_scf(c, p, b)
    torch.cuda.synchronize()
    b.close()
    clocks = sampler.stop()
    if not r.converged:
        raise RuntimeError("the learned+mixed Si216 run did not reach the target")
    fp64_s, mixed_s = float(hit[3]), float(r.wall_s)
    mhz = clocks.get("sm_mhz") or None
    return {
        "workload": "Si216 3x3x3 conventional, sigma 0.05 A (seed 3), 25 Ry, 108^3, Gamma, 448 bands, LDA-PZ, fixed occupations",
        "criterion": "|E - E_target| < 1e-6 Ry/atom, E_target = plain FP64 run to density RMS residual 1e-8",
        "target_energy_per_atom": ref.energy / natom,
        "fp64": {"seconds": round(fp64_s, 3), "scf_iterations": int(hit[0]),
                 "dE_per_atom": (hit[1] - ref.energy) / natom, "run_to_target_seconds": round(ref.wall_s, 3),
                 "run_to_target_iterations": ref.iterations},
        "learned_mixed": {"seconds": round(mixed_s, 3), "scf_iterations": r.iterations,
                          "dE_per_atom": (r.energy - ref.energy) / natom,
                          "switched_to_fp64_at_iteration": getattr(b, "switched_at", None),
                          "precision": "TF32X3 contexts (FP32 FFT passes, 3xTF32 tensor-core GEMMs) + MLP preconditioner, FP64 after the switch"},
        "speedup_vs_fp64": round(fp64_s / mixed_s, 3),
        "clocks": clocks,
        "seconds_x_median_sm_ghz": {"fp64": round(fp64_s * mhz / 1e3, 3), "learned_mixed": round(mixed_s * mhz / 1e3, 3)} if mhz else None,
    }


def run_profile_case(precision: str = "fp64", cell: str = "si64"):
    """One k-point (Gamma) of a benchmark cell, a few columns, H|psi> twice and one band-density
    accumulation of the same columns: a small case for ncu captures of single kernels (Si64: 32
    columns, a few hundred MB on the device; Si216: 16 columns, under 1 GB)."""
    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    import importlib

    system = importlib.import_module("dftzig_b200.system")
    w = WORKLOADS[cell]
    ncols = 32 if cell == "si64" else 16
    c = system.crystal(w["cell"], w["seed"])
    dims = system.fft_box(w["ecut"], c.recip)
    inp = system.kpoint_inputs(c, w["ecut"], (0.0, 0.0, 0.0), dims=dims)
    prec = {"fp64": dz.PRECISION_FP64, "fp32": dz.PRECISION_FP32, "tf32": dz.PRECISION_TF32}[precision]
    kc = dz.KpointContext(dims[0], dims[1], dims[2], inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, prec)
    kc.set_vloc(inp.local_r)
    kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
    x = torch.randn((ncols, kc.n), dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        kc.apply_hamiltonian_async(x, y, ncols, s.cuda_stream)
    torch.cuda.synchronize()
    rho = torch.zeros(dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
    kc.accumulate_band_density(x, np.full(ncols, 2.0), rho)
    torch.cuda.synchronize()
    kc.close()
    print("profile case done", flush=True)


def run_scf_workload(args):
    """Time-to-SCF on Si2 (FCC primitive, a = 5.431 A), 20 Ry, 20^3 box, 4x4x4 Gamma-centred MP mesh
    folded by time reversal (36 k-points), 8 bands, fixed occupations, Pulay 8 / beta 0.3 potential
    mixing, the reference's default eigensolver settings (tol 1e-4, 20 iterations, 2 warm-up
    iterations at 1e-3 / 10) and warm starts.  Target energy: a tight FP64 run on the same device
    (density RMS 1e-9, eigensolver tol 1e-10).  Reported: wall seconds until |E - E_target| < 1e-6
    Ry/atom, plain FP64 and mixed (FP32 FFT passes until the density residual < 1e-5)."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si2")
    base = dict(ecut=20.0, kmesh=(4, 4, 4), nbands=8, mixing_beta=0.3, pulay_history=8, max_iter=60)
    tight = scf.ScfParams(**base, convergence=1e-9, iterative_tol=1e-10, iterative_max_iter=200, warmup_steps=0)
    b = scf.GpuBackend(dz, "fp64")
    ref = scf.run_scf(c, tight, b)
    b.close()
    out = {}
    for mode in ("fp64", "mixed"):
        p = scf.ScfParams(**base, convergence=1e-12, energy_target=ref.energy, energy_tol_per_atom=1e-6)
        times = []
        its = []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            b = scf.GpuBackend(dz, mode)
            r = scf.run_scf(c, p, b)
            torch.cuda.synchronize()
            b.close()
            times.append(r.wall_s)
            its.append(r.iterations)
            if not r.converged:
                raise RuntimeError(f"time-to-SCF run ({mode}) did not reach the target")
        out[mode] = (float(np.median(times)), int(np.median(its)))
    line = {
        "metric": "time-to-SCF (|dE| < 1e-6 Ry/atom vs tight FP64), Si2 20 Ry 4x4x4",
        "value": round(out["mixed"][0], 3),
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": 1,
        "steps": max(1, args.steps),
        "dtype": "f64/f32",
        "data": "synthetic (synthetic GTH-form Si pseudopotential)",
        "config": {"workload": "Si2 FCC 5.431 A, 20 Ry, 20^3, 4x4x4 MP (36 k, time-reversal folded), 8 bands, fixed occupations, Pulay 8 beta 0.3",
                   "target_energy_per_atom": ref.energy_per_atom, "target_iterations": ref.iterations},
        "fp64": {"seconds": round(out["fp64"][0], 3), "scf_iterations": out["fp64"][1]},
        "mixed": {"seconds": round(out["mixed"][0], 3), "scf_iterations": out["mixed"][1], "switch": "FP32 FFT passes until drho < 1e-5, then FP64"},
    }
    print(json.dumps(line), flush=True)


def run_scf216_workload(args):
    """Time-to-SCF on Si216 (3x3x3 conventional, N(0, 0.05 A) displacements, seed 3), 25 Ry, Gamma
    only, 448 bands, LDA-PZ, fixed occupations, Pulay 8 / beta 0.3, the reference's eigensolver
    defaults (max_subspace 4 nb + 8 = 1800).  Target: a tight FP64 run (density RMS 1e-8).  Reported:
    wall seconds until |E - E_target| < 1e-6 Ry/atom, plain FP64 (reference preconditioner) against
    learned+mixed (TF32X3 contexts until the density residual is below 1e-4, then FP64; the trained
    TPA-refining MLP preconditioner throughout).  Both runs use the resident driver (eigenvectors,
    density, Hartree-XC potential and Pulay history on the device)."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    learn = importlib.import_module("dftzig_b200.learn")
    c = system.crystal("si216", 3)
    base = dict(ecut=25.0, kmesh=(1, 1, 1), nbands=448, mixing_beta=0.3, pulay_history=8, max_iter=60)
    b = scf.GpuBackend(dz, "fp64", resident=True)
    ref = scf.run_scf(c, scf.ScfParams(**base, convergence=1e-8), b)
    b.close()
    mlp = (dz.PRECOND_MLP, learn.load_precond_weights())
    out = {}
    for mode, prec, pc in (("fp64", "fp64", None), ("learned_mixed", "mixed", mlp)):
        p = scf.ScfParams(**base, convergence=1e-12, energy_target=ref.energy, energy_tol_per_atom=1e-6)
        torch.cuda.synchronize()
        # resident: eigenvectors, density, potential and Pulay history stay on the device
        b = scf.GpuBackend(dz, prec, precond=pc, resident=True, switch_drho=args.switch_drho)
        r = scf.run_scf(c, p, b)
        torch.cuda.synchronize()
        b.close()
        if not r.converged:
            raise RuntimeError(f"time-to-SCF run ({mode}) did not reach the target")
        out[mode] = {"seconds": round(r.wall_s, 3), "scf_iterations": r.iterations, "dE_per_atom": r.energy_per_atom - ref.energy_per_atom,
                     "switched_to_fp64_at_iteration": getattr(b, "switched_at", None),
                     # per SCF iteration: seconds since start, density residual, solver precision,
                     # Davidson iterations, H applications
                     "trace": [[round(h[3], 2), float(f"{h[2]:.2e}"), sv[0], sv[1], sv[2]] for h, sv in zip(r.history, b.solves)]}
    line = {
        "metric": "time-to-SCF (|dE| < 1e-6 Ry/atom vs tight FP64), Si216 25 Ry Gamma, learned+mixed vs plain FP64",
        "value": out["learned_mixed"]["seconds"],
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": 1,
        "steps": 1,
        "dtype": "f64/f32/tf32x3",
        "data": "synthetic (seeded displacements; synthetic GTH-form Si pseudopotential)",
        "config": {"workload": "Si216 3x3x3 conventional, sigma 0.05 A (seed 3), 25 Ry, Gamma, 448 bands, fixed occupations",
                   "switch_drho": args.switch_drho,
                   "target_energy_per_atom": ref.energy_per_atom, "target_iterations": ref.iterations, "target_seconds": round(ref.wall_s, 3)},
        "fp64": out["fp64"],
        "learned_mixed": out["learned_mixed"],
        "speedup_vs_fp64": round(out["fp64"]["seconds"] / out["learned_mixed"]["seconds"], 3),
    }
    print(json.dumps(line), flush=True)


def run_scf64_workload(args):
    """Time-to-SCF on Si64 (2x2x2 conventional, N(0, 0.02 A) displacements, seed 1), 30 Ry, 75^3,
    2x2x2 MP (8 k), 160 bands, Fermi-Dirac 0.01 Ry, PBE (--xc lda for LDA-PZ), Pulay 8 / beta 0.3,
    the reference's eigensolver defaults, the resident driver.  Target: a tight FP64 run (density
    RMS 1e-8).  Reported: wall seconds until |E - E_target| < 1e-6 Ry/atom, plain FP64 and mixed
    (TF32X3 contexts until the density residual is below 1e-4 or stalls, then FP64), with each run's
    largest force and eigenvalue error against the tight FP64 run."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si64", 1)
    base = dict(ecut=30.0, kmesh=(2, 2, 2), nbands=160, mixing_beta=0.3, pulay_history=8, max_iter=60, smearing=0.01, xc=args.xc)
    b = scf.GpuBackend(dz, "fp64", resident=True)
    ref = scf.run_scf(c, scf.ScfParams(**base, convergence=1e-8), b, forces=True)
    b.close()
    out = {}
    errs = {}
    for mode in ("fp64", "mixed"):
        p = scf.ScfParams(**base, convergence=1e-12, energy_target=ref.energy, energy_tol_per_atom=1e-6)
        torch.cuda.synchronize()
        b = scf.GpuBackend(dz, mode, resident=True)
        r = scf.run_scf(c, p, b, forces=True)  # forces after the timed loop (not in wall_s)
        torch.cuda.synchronize()
        b.close()
        if not r.converged:
            raise RuntimeError(f"time-to-SCF run ({mode}) did not reach the target")
        out[mode] = (r.wall_s, r.iterations, r.energy_per_atom - ref.energy_per_atom, getattr(b, "switched_at", None))
        nb = min(len(ref.eigenvalues[0]), len(r.eigenvalues[0]))
        errs[mode] = {"force_error_max_ry_per_bohr": float(np.abs(r.forces - ref.forces).max()),
                      "eigenvalue_error_max_ry": float(max(np.abs(np.asarray(a)[:nb] - np.asarray(e)[:nb]).max()
                                                           for a, e in zip(r.eigenvalues, ref.eigenvalues)))}
    line = {
        "metric": "time-to-SCF (|dE| < 1e-6 Ry/atom vs tight FP64), Si64 30 Ry 2x2x2, mixed precision",
        "value": round(out["mixed"][0], 3),
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": 1,
        "steps": 1,
        "dtype": "f64/f32/tf32x3",
        "data": "synthetic (seeded displacements; synthetic GTH-form Si pseudopotential)",
        "config": {"workload": f"Si64 2x2x2 conventional, sigma 0.02 A (seed 1), 30 Ry, 75^3, 2x2x2 MP (8 k), 160 bands, FD 0.01 Ry, {args.xc.upper()}",
                   "target_energy_per_atom": ref.energy_per_atom, "target_iterations": ref.iterations},
        "fp64": {"seconds": round(out["fp64"][0], 3), "scf_iterations": out["fp64"][1], "dE_per_atom": out["fp64"][2], **errs["fp64"]},
        "mixed": {"seconds": round(out["mixed"][0], 3), "scf_iterations": out["mixed"][1], "dE_per_atom": out["mixed"][2],
                  "switched_to_fp64_at_iteration": out["mixed"][3], **errs["mixed"]},
        "reference_max_force_ry_per_bohr": float(np.abs(ref.forces).max()),
        "speedup_mixed_vs_fp64": round(out["fp64"][0] / out["mixed"][0], 3),
    }
    print(json.dumps(line), flush=True)


def run_al4_workload(args):
    """Config 3: batched uneven k-points.  FCC Al conventional cell (a = 4.05 A, seeded symmetric
    strain in [-1%, 1%], seed 2), LDA-PZ, 25 Ry, 27^3 box, the full 8x8x8 Monkhorst-Pack mesh folded by
    time reversal (260 k-points, plane-wave counts differing from k-point to k-point), 12 bands,
    Fermi-Dirac 0.02 Ry, Pulay 8 / beta 0.3, the reference's eigensolver defaults, resident driver.
    Every SCF iteration solves all k-points in one lockstep batch (dftcuda_eig_solve_batch).  Target:
    the plain FP64 run carried on to a density residual of 1e-8; reported: wall seconds to
    |E - E_target| < 1e-6 Ry/atom for plain FP64 (from its own trajectory) and for mixed precision
    (TF32X3 contexts, FP64 after the switch), k-point solves per second, and the host-side phases."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("al4", 2)
    natom = len(c.atom_species)
    base = dict(ecut=25.0, kmesh=(8, 8, 8), nbands=12, smearing=0.02, mixing_beta=0.3, pulay_history=8, max_iter=80)
    kpts = system.monkhorst_pack(base["kmesh"])
    npws = [system.basis(c.recip, base["ecut"], k).hkl.shape[0] for k, _ in kpts]
    sampler = ClockSampler(0)
    sampler.start()
    torch.cuda.synchronize()
    b = scf.GpuBackend(dz, "fp64", resident=True)
    ref = scf.run_scf(c, scf.ScfParams(**base, convergence=1e-8), b)
    torch.cuda.synchronize()
    b.close()
    hit = next(h for h in ref.history if abs(h[1] - ref.energy) / natom < 1e-6)
    p = scf.ScfParams(**base, convergence=1e-12, energy_target=ref.energy, energy_tol_per_atom=1e-6)
    b = scf.GpuBackend(dz, "mixed", resident=True)
    r = scf.run_scf(c, p, b)
    torch.cuda.synchronize()
    b.close()
    clocks = sampler.stop()
    line = {
        "metric": "time-to-SCF (|dE| < 1e-6 Ry/atom vs tight FP64), Al4 25 Ry 8x8x8 (260 k-points), batched",
        "value": round(float(hit[3]), 3),
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": 1,
        "steps": 1,
        "dtype": "f64 (mixed: f32 FFT passes + 3xTF32 GEMMs, FP64 after the switch)",
        "data": "synthetic (seeded strain; synthetic GTH-form Al pseudopotential)",
        "config": {"workload": "Al4 FCC conventional 4.05 A, strain +-1% (seed 2), LDA-PZ, 25 Ry, 27^3, 8x8x8 MP (k/-k folded), 12 bands, FD 0.02 Ry",
                   "kpoints": len(kpts), "n_pw_min": int(min(npws)), "n_pw_max": int(max(npws)),
                   "target_energy_per_atom": ref.energy_per_atom},
        "fp64": {"seconds": round(float(hit[3]), 3), "scf_iterations": int(hit[0]), "run_to_target_seconds": round(ref.wall_s, 3),
                 "kpoint_solves_per_second": round(len(kpts) * int(hit[0]) / float(hit[3]), 1)},
        "mixed": {"seconds": round(r.wall_s, 3), "scf_iterations": r.iterations, "dE_per_atom": (r.energy - ref.energy) / natom,
                  "switched_to_fp64_at_iteration": getattr(b, "switched_at", None),
                  "kpoint_solves_per_second": round(len(kpts) * r.iterations / r.wall_s, 1)},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_cells_workload(args):
    """Many-cell SCF throughput on seeded SiGe8 cells (x ~ U(0,1), Vegard lattice 5.43-5.66 A,
    +-2% strain; seeds 2400..), 20 Ry, 2x2x2 MP, 20 bands, FD 0.005 Ry: all cells' k-points go
    through one lockstep eigensolver batch per SCF iteration, with the resident driver (each cell's
    eigenvectors, density, potential and mixing on the device).  Atomic-superposition start against
    the learned (FNO) start; cells per second = cells / wall time to convergence (RMS drho 1e-6)."""
    import importlib

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    learn = importlib.import_module("dftzig_b200.learn")
    cells = [system.crystal("sige8", 2400 + i) for i in range(args.cells)]
    ecut = 20.0
    p = scf.ScfParams(ecut=ecut, kmesh=(2, 2, 2), nbands=20, convergence=1e-6, max_iter=80, smearing=learn.FNO_SMEARING)
    names = [s for s in args.cells_starts.split(",") if s in ("atomic", "fno")]
    starts = {"atomic": [], "fno": []}
    params = learn.load_fno_weights()
    for c in cells:
        dims, u, rho_at, mean = learn.fno_input(c, ecut)
        if "atomic" in names:
            starts["atomic"].append(rho_at * (c.nelec / (rho_at.mean() * c.volume)))
        if "fno" in names:
            starts["fno"].append(learn.fno_initial_density(dz, params, c, ecut))
    out = {}
    for name in names:
        # the learned start skips the loose-tolerance warm-up iterations meant for poor densities
        pn = p if name == "atomic" else scf.ScfParams(**{**p.__dict__, "warmup_steps": 0})
        res, wall = scf.run_scf_many(dz, cells, pn, "fp64", starts[name], resident=True)
        out[name] = {"seconds": round(wall, 3), "cells_per_second": round(len(cells) / wall, 3),
                     "phases_s": getattr(scf.run_scf_many, "last_phases", None),
                     "mean_scf_iterations": float(np.mean([r.iterations for r in res])),
                     "all_converged": all(r.converged for r in res)}
    line = {
        "metric": "many-cell SCF throughput (cells/s), SiGe8 20 Ry 2x2x2, learned FNO start",
        "value": out["fno" if "fno" in out else names[0]]["cells_per_second"],
        "unit": "cells/s",
        "higher_is_better": True,
        "n_gpus": 1,
        "steps": 1,
        "dtype": "f64 (FNO f32)",
        "data": "synthetic seeded SiGe8 cells (synthetic GTH-form Si and Ge pseudopotentials)",
        "config": {"workload": f"{len(cells)} SiGe8 cells, 20 Ry, 2x2x2 MP (8 k), 20 bands, FD 0.005 Ry, lockstep batch", "cells": len(cells)},
        "atomic_start": out.get("atomic"),
        "fno_start": out.get("fno"),
    }
    print(json.dumps(line), flush=True)


def run_eig_workload(args):
    """One Davidson solve at Gamma from the random start, --eig-iters iterations: the Si64 cell (30 Ry,
    160 bands) or the Si216 cell (25 Ry, 448 bands, subspace up to 1800); --precision selects the
    context precision.  The case the eigensolver's launch lists are taken on."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    system = importlib.import_module("dftzig_b200.system")
    cell, seed, ecut, nb = (CELL, SEED, ECUT, NBANDS) if args.eig_cell == "si64" else ("si216", 3, 25.0, 448)
    c = system.crystal(cell, seed)
    inp = system.kpoint_inputs(c, ecut, (0.0, 0.0, 0.0))
    prec = {"fp64": dz.PRECISION_FP64, "fp32": dz.PRECISION_FP32, "tf32": dz.PRECISION_TF32X3}[args.precision]
    kc = dz.KpointContext(*inp.dims, inp.volume, inp.basis.hkl, inp.basis.kinetic, inp.basis.gcart, prec)
    kc.set_vloc(inp.local_r)
    kc.set_projectors([dz.SpeciesProjectors(l, d, p) for (l, d, p) in inp.species_phi], inp.atom_species, inp.positions)
    if args.eig_precond == "tpa":
        kc.set_preconditioner(dz.PRECOND_TPA)
    elif args.eig_precond == "mlp":
        kc.set_preconditioner(dz.PRECOND_MLP, importlib.import_module("dftzig_b200.learn").load_precond_weights())
    kc.set_profiling(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = kc.hermitian_eigen_decomp_iterative(inp.basis.kinetic, nb, dz.Options(max_iter=args.eig_iters, tol=args.eig_tol))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    pr = kc.profile()
    kc.close()
    print(json.dumps({"metric": f"Davidson solve wall time, {cell} Gamma {ecut:g} Ry {nb} bands ({args.precision})", "value": round(wall * 1e3, 2), "unit": "ms",
                      "preconditioner": args.eig_precond, "tol": args.eig_tol, "converged": bool(r.converged),
                      "iterations": r.iterations, "h_applies": r.h_applies, "apply_h_ms": round(pr["apply_h_ns"] / 1e6, 2),
                      "subspace_ms": round(pr["subspace_ns"] / 1e6, 2)}), flush=True)


def run_potential_workload(args):
    """The SCF potential kernels on the Si216 box (108^3, 1,259,712 points): the Hartree + LDA-PZ
    build from a seeded density (dftcuda_hxc_potential), V(r) = V_loc + FFT^-1 V(G)
    (dftcuda_potential_real), one Pulay step on the complex V(G) with a full 8-deep history
    (dftcuda_pulay_mix), and the standalone forward + inverse 3D FFT (dftcuda_fft3d).  Device-resident
    torch tensors; CUDA-event time of each call after warm-up, median of five.  Bytes per call are
    the arrays each call must read and write once (N points: density 8 B, V(G) 16 B, V(r) 8 B)."""
    import importlib

    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("si216", 3)
    dims = system.fft_box(25.0, c.recip)
    N = dims[0] * dims[1] * dims[2]
    gen = torch.Generator(device="cuda").manual_seed(0)
    rho = (c.nelec / c.volume) * (1.0 + 0.1 * torch.rand(N, dtype=torch.float64, device="cuda", generator=gen))
    vloc = torch.randn(N, dtype=torch.float64, device="cuda", generator=gen)
    pot = dz.PotentialContext(dims, c.volume, c.recip, history=8, functional="lda")
    plan = dz.Fft3dPlan(*dims)
    vg, _ = pot.hxc(rho)
    x = torch.view_as_real(vg).reshape(-1).clone()
    for _ in range(8):  # fill the history
        pot.pulay_mix(x, 1e-3 * torch.randn(2 * N, dtype=torch.float64, device="cuda", generator=gen), 0.3)
    box = torch.randn(N, dtype=torch.complex128, device="cuda", generator=gen)
    resid = 1e-3 * torch.randn(2 * N, dtype=torch.float64, device="cuda", generator=gen)

    def timed(fn):
        fn()
        ts = []
        for _ in range(5):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    rows = {}
    for name, fn, nbytes in (
            ("hxc_lda", lambda: pot.hxc(rho, v_in=vg, out=vg), N * (8 + 16 + 16)),
            ("potential_real", lambda: pot.real(vg, vloc=vloc), N * (16 + 8 + 8)),
            ("pulay_mix_h8", lambda: pot.pulay_mix(x, resid, 0.3), N * 16 * (2 * 8 + 3)),
            ("fft3d_fwd_inv", lambda: (plan.forward(box), plan.inverse(box)), N * 16 * 4)):
        ms = timed(fn)
        rows[name] = {"ms": round(ms, 4), "bytes": int(nbytes), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1)}
    pot.close()
    plan.close()
    print(json.dumps({"workload": f"Si216 box {dims[0]}x{dims[1]}x{dims[2]}, potential kernels", "calls": rows}), flush=True)


def run_heev_workload(args):
    """The subspace eigensolver (dftcuda_hermitian_eigen_decomp: tridiagonalisation, bisection,
    inverse iteration, WY back-transformation) on a seeded random Hermitian m x m matrix, lowest m/3
    pairs: device time of two calls after one warm-up, and the eigenvalue error against LAPACK."""
    import torch

    import dftzig_loader

    dz = dftzig_loader.load()
    lib = dz.load_library()
    m = args.heev_m
    nev = max(1, m // 3)
    rng = np.random.default_rng(m)
    x = rng.normal(size=(m, m)) + 1j * rng.normal(size=(m, m))
    a = 0.05 * (x + x.conj().T) / 2
    at = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    vals = torch.empty(nev, dtype=torch.float64, device="cuda")
    vecs = torch.empty((nev, m), dtype=torch.complex128, device="cuda")
    ms = []
    for rep in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = lib.dftcuda_hermitian_eigen_decomp(m, at.data_ptr(), nev, vals.data_ptr(), vecs.data_ptr())
        torch.cuda.synchronize()
        if st != 0:
            raise RuntimeError(f"hermitian_eigen_decomp failed ({st})")
        ms.append(1e3 * (time.perf_counter() - t0))
    err = float(np.abs(vals.cpu().numpy() - np.linalg.eigvalsh(a)[:nev]).max())
    print(json.dumps({"metric": f"subspace eigensolver wall time, m = {m}, lowest {nev} pairs", "value": round(min(ms[1:]), 2),
                      "unit": "ms", "eigenvalue_error_max": err}), flush=True)


def run_scf216_kernel_table(args):
    """The first --profile-steps SCF steps of both Si216 arms under torch.profiler (CUPTI activity
    records): per arm, the GPU time of each kernel summed over the steps, and the wall time."""
    import importlib

    import torch
    from torch.profiler import ProfilerActivity, profile

    import dftzig_loader

    dz = dftzig_loader.load()
    scf = importlib.import_module("dftzig_b200.scf")
    system = importlib.import_module("dftzig_b200.system")
    learn = importlib.import_module("dftzig_b200.learn")
    c = system.crystal("si216", 3)
    base = dict(ecut=25.0, kmesh=(1, 1, 1), nbands=448, mixing_beta=0.3, pulay_history=8, max_iter=args.profile_steps)
    mlp = (dz.PRECOND_MLP, learn.load_precond_weights())
    out = {}
    for mode, prec, pc in (("fp64", "fp64", None), ("learned_mixed", "mixed", mlp)):
        b = scf.GpuBackend(dz, prec, precond=pc, resident=True, switch_drho=args.switch_drho)
        t0 = time.perf_counter()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            scf.run_scf(c, scf.ScfParams(**base, convergence=1e-12), b)
            torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        b.close()
        rows = []
        for e in prof.key_averages():
            t = getattr(e, "device_time_total", 0) or getattr(e, "cuda_time_total", 0)
            if t > 0:
                rows.append((round(t / 1e3, 1), e.count, e.key.replace("(anonymous namespace)::", "").split("(")[0][:80]))
        rows.sort(reverse=True)
        out[mode] = {"wall_s": round(wall, 2), "gpu_kernel_ms": round(sum(r[0] for r in rows), 1), "davidson": b.solves,
                     "top": [{"ms": r[0], "launches": r[1], "kernel": r[2]} for r in rows[:20]]}
    print(json.dumps({"metric": f"Si216 kernel-time table, first {args.profile_steps} SCF steps", **out}), flush=True)


def main():
    args = parse()
    if args.workload == "gemm":
        return run_gemm_workload(args)
    if args.workload == "potential":
        return run_potential_workload(args)
    if args.workload == "heev":
        run_heev_workload(args)
        return
    if args.workload == "scf216" and args.profile_steps > 0:
        run_scf216_kernel_table(args)
        return
    if args.workload == "eig":
        run_eig_workload(args)
        return
    if args.workload == "scf":
        run_scf_workload(args)
        return
    if args.workload == "scf64":
        run_scf64_workload(args)
        return
    if args.workload == "scf216":
        run_scf216_workload(args)
        return
    if args.workload == "cells":
        run_cells_workload(args)
        return
    if args.workload == "al4":
        run_al4_workload(args)
        return
    if args.profile_case:
        run_profile_case(args.precision, args.cell)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
