"""k-point parallel SCF (dft-zig_b200/kpar.py): two ranks, each solving its share of the k-points,
reproduce the one-process run.  On the CPU with the oracle backend over gloo; on the GPU with
libdftcuda contexts (two processes sharing one device) over gloo."""
import importlib
import os
import socket
import tempfile

import numpy as np
import pytest

import dftzig_loader

dftzig_loader.load()
scf = importlib.import_module("dftzig_b200.scf")
system = importlib.import_module("dftzig_b200.system")
kpar = importlib.import_module("dftzig_b200.kpar")

CASES = {
    # fixed occupations: only the density crosses ranks
    "fixed": dict(ecut=8.0, kmesh=(2, 2, 2), nbands=8, convergence=1e-8, iterative_max_iter=100, iterative_tol=1e-9, warmup_steps=0),
    # Fermi-Dirac smearing: the Fermi level needs every rank's eigenvalues
    "smeared": dict(ecut=8.0, kmesh=(2, 2, 1), nbands=8, convergence=1e-8, iterative_max_iter=100, iterative_tol=1e-9, warmup_steps=0,
                    smearing=0.01),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, backend="oracle", cases=None):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import datetime

    import torch.distributed as dist

    import dftzig_loader as dl

    dl.load()
    sc = importlib.import_module("dftzig_b200.scf")
    sy = importlib.import_module("dftzig_b200.system")
    kp = importlib.import_module("dftzig_b200.kpar")
    from tests.helpers import OracleBackend

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        comm = kp.KpointComm()
        for name, kw in (cases or CASES).items():
            st_backend = OracleBackend() if backend == "oracle" else sc.GpuBackend(dl.load())
            r = sc.run_scf(sy.crystal("si2"), sc.ScfParams(**kw), st_backend, comm=comm)
            np.savez(os.path.join(out_dir, f"{name}_{rank}.npz"), energy=r.energy, iterations=r.iterations,
                     values=np.array(r.eigenvalues), rho=r.rho, nlocal=len(st_backend.ctxs))
            if backend != "oracle":
                st_backend.close()
    finally:
        dist.destroy_process_group()


def test_deal_kpoints_balances_and_covers():
    owner = kpar.deal_kpoints(8, 3)
    assert sorted(set(owner)) == [0, 1, 2] and len(owner) == 8
    assert owner == sorted(owner)  # contiguous blocks
    costs = [100, 90, 80, 70, 60, 50, 40, 30]
    owner = kpar.deal_kpoints(8, 2, costs)
    load = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(2)]
    assert abs(load[0] - load[1]) <= 10
    assert kpar.deal_kpoints(5, 1) == [0] * 5
    assert kpar.deal_kpoints(2, 4) == [0, 2]  # more ranks than k-points: some ranks idle


def _check_two_ranks(backend, make_backend, cases, e_tol, v_tol, rho_rtol):
    import torch.multiprocessing as mp

    serial = {}
    for name, kw in cases.items():
        b = make_backend()
        serial[name] = scf.run_scf(system.crystal("si2"), scf.ScfParams(**kw), b)
        if hasattr(b, "close"):
            b.close()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d, backend, cases), nprocs=2, join=True, start_method="spawn")
        for name in cases:
            r0 = np.load(os.path.join(d, f"{name}_0.npz"))
            r1 = np.load(os.path.join(d, f"{name}_1.npz"))
            s = serial[name]
            nk = len(system.monkhorst_pack(cases[name]["kmesh"]))
            assert int(r0["nlocal"]) + int(r1["nlocal"]) == nk and int(r0["nlocal"]) > 0 and int(r1["nlocal"]) > 0
            # the replicated state is bit-identical on both ranks
            assert float(r0["energy"]) == float(r1["energy"])
            np.testing.assert_array_equal(r0["rho"], r1["rho"])
            np.testing.assert_array_equal(r0["values"], r1["values"])
            # and matches the one-process run up to the order of the density sum
            assert abs(int(r0["iterations"]) - s.iterations) <= (0 if backend == "oracle" else 1)
            assert abs(float(r0["energy"]) - s.energy) < e_tol
            np.testing.assert_allclose(r0["values"], np.array(s.eigenvalues), atol=v_tol)
            np.testing.assert_allclose(r0["rho"], s.rho, atol=rho_rtol * float(np.abs(s.rho).max()))


def test_two_rank_kpoint_scf_matches_one_process():
    from tests.helpers import OracleBackend

    _check_two_ranks("oracle", OracleBackend, CASES, 1e-10, 1e-9, 1e-10)


def test_rank_without_kpoints_follows_the_run():
    """Gamma only on two ranks: rank 1 owns no k-point, builds no context and solves nothing, yet
    takes part in every reduction and ends with the same state as rank 0 and the one-process run."""
    import torch.multiprocessing as mp

    from tests.helpers import OracleBackend

    cases = {"gamma": dict(CASES["fixed"], kmesh=(1, 1, 1))}
    s = scf.run_scf(system.crystal("si2"), scf.ScfParams(**cases["gamma"]), OracleBackend())
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d, "oracle", cases), nprocs=2, join=True, start_method="spawn")
        r0 = np.load(os.path.join(d, "gamma_0.npz"))
        r1 = np.load(os.path.join(d, "gamma_1.npz"))
    assert int(r0["nlocal"]) == 1 and int(r1["nlocal"]) == 0
    assert float(r0["energy"]) == float(r1["energy"])
    np.testing.assert_array_equal(r0["rho"], r1["rho"])
    np.testing.assert_array_equal(r0["values"], r1["values"])
    assert int(r0["iterations"]) == s.iterations
    assert abs(float(r0["energy"]) - s.energy) < 1e-12
    np.testing.assert_allclose(r0["values"], np.array(s.eigenvalues), atol=1e-12)


@pytest.mark.gpu
def test_two_rank_kpoint_scf_on_gpu_matches_one_process(dz):
    """The same split with libdftcuda contexts: two processes share the one GPU, each holding the
    contexts of its own k-points (the kernels of the two ranks never wait on each other), and the
    density and eigenvalues cross through gloo on the host."""
    cases = {"fixed": dict(CASES["fixed"], convergence=1e-7)}
    _check_two_ranks("gpu", lambda: scf.GpuBackend(dz), cases, 1e-8, 1e-7, 1e-7)
