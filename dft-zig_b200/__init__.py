"""dft-zig B200 hot path: host-side mirror of the reference interfaces over libdftcuda.so.

The CUDA work all happens in ``libdftcuda.so`` (built from ``csrc/`` by ``build.py``); this module only
binds its C ABI (``include/dftcuda.h``) with ctypes and mirrors the reference's names:

  KpointContext.apply_hamiltonian(_batched)  src/features/scf/apply.zig:643-658, 1584-1618
  Options / hermitian_eigen_decomp_iterative src/features/linalg/lobpcg/common.zig:44-52,
                                             src/features/linalg/iterative.zig:67-76
  KpointContext.accumulate_band_density      src/features/scf/kpoint/density.zig:444-474
  KpointContext.nonlocal_energies            src/features/scf/kpoint/density.zig:238-266
  Fft3dPlan.forward / inverse                src/features/fft/fft.zig:224-263 (FFTW semantics)

Errors raise exceptions named after the reference's Zig errors (InvalidMatrixSize, InvalidGrid,
LapackFailure, ...).  There is no CPU fallback: without the built library, or without a CUDA
device, every entry point raises.

Arrays: numpy arrays are host memory (the call copies through the library's device buffers);
torch CUDA tensors are passed as device pointers.  Blocks of vectors are ``(ncols, n)``
complex128 C-contiguous arrays, i.e. the reference's column-major [n x ncols] layout.
"""
from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdftcuda.so")

# C-ABI symbols declared in include/dftcuda.h (checked by tests/test_abi.py).
ABI_SYMBOLS = (
    "dftcuda_status_string",
    "dftcuda_last_error_message",
    "dftcuda_device_count",
    "dftcuda_debug_set_wait_limits",
    "dftcuda_debug_fail_alloc",
    "dftcuda_fermi_occupations",
    "dftcuda_ionic_potential_radial",
    "dftcuda_nonlocal_stress",
    "dftcuda_local_forces_radial",
    "dftcuda_kctx_create",
    "dftcuda_kctx_destroy",
    "dftcuda_kctx_npw",
    "dftcuda_set_vloc",
    "dftcuda_set_projectors",
    "dftcuda_apply_h_batch",
    "dftcuda_apply_h",
    "dftcuda_apply_h_batch_async",
    "dftcuda_nonlocal_energies",
    "dftcuda_eig_solve",
    "dftcuda_accumulate_density",
    "dftcuda_fft_plan_create",
    "dftcuda_fft_plan_destroy",
    "dftcuda_fft3d",
    "dftcuda_kctx_set_profiling",
    "dftcuda_kctx_get_profile",
    "dftcuda_accumulate_density_noalloc",
    "dftcuda_hermitian_eigen_decomp",
    "dftcuda_eig_solve_batch",
    "dftcuda_kctx_autotune",
    "dftcuda_kctx_set_preconditioner",
    "dftcuda_precond_mlp_loss_grad",
    "dftcuda_precond_mlp_train",
    "dftcuda_fno_forward",
    "dftcuda_fno_loss_grad",
    "dftcuda_fno_train",
    "dftcuda_complex_gemm",
    "dftcuda_pctx_create",
    "dftcuda_pctx_destroy",
    "dftcuda_hxc_potential",
    "dftcuda_potential_real",
    "dftcuda_pulay_mix",
    "dftcuda_pulay_reset",
    "dftcuda_ionic_potential",
    "dftcuda_pctx_set_functional",
    "dftcuda_local_forces",
    "dftcuda_nonlocal_forces",
    "dftcuda_radial_table",
    "dftcuda_plane_wave_basis",
    "dftcuda_projector_phi",
    "dftcuda_symmetrize_density",
)

PRECOND_REFERENCE = 0  # r / (|k+G|^2 - lambda), lobpcg/common.zig:214-226
PRECOND_TPA = 1  # Teter-Payne-Allan
PRECOND_MLP = 2  # learned per-plane-wave MLP
PRECOND_MLP_PARAMS = 4481
FNO_PARAMS = 2097473  # learned first SCF density (Fourier neural operator)

PRECISION_FP64 = 0
PRECISION_FP32 = 1
PRECISION_TF32 = 2  # FP32 FFT passes + tcgen05 TF32 projector GEMMs (~1e-3)
PRECISION_TF32X3 = 3  # FP32 FFT passes + split (3xTF32) tensor-core GEMMs (~1e-6)


class DftCudaError(RuntimeError):
    status = -5


class InvalidMatrixSize(DftCudaError):
    status = -1


class InvalidGrid(DftCudaError):
    status = -2


class LapackFailure(DftCudaError):
    status = -3


class OutOfMemory(DftCudaError):
    status = -4


class CudaError(DftCudaError):
    status = -5


class InvalidArgument(DftCudaError):
    status = -6


class Unsupported(DftCudaError):
    status = -7


class Timeout(DftCudaError):
    status = -8


_ERRORS = {c.status: c for c in (InvalidMatrixSize, InvalidGrid, LapackFailure, OutOfMemory, CudaError, InvalidArgument, Unsupported, Timeout)}


class _Species(ct.Structure):
    _fields_ = [
        ("beta_count", ct.c_size_t),
        ("l_list", ct.POINTER(ct.c_int32)),
        ("dij", ct.POINTER(ct.c_double)),
        ("m_total", ct.c_size_t),
        ("phi", ct.POINTER(ct.c_double)),
    ]


class _EigOpts(ct.Structure):
    _fields_ = [
        ("max_iter", ct.c_size_t),
        ("tol", ct.c_double),
        ("max_subspace", ct.c_size_t),
        ("block_size", ct.c_size_t),
        ("init_diagonal", ct.c_int),
    ]


class _EigInfo(ct.Structure):
    _fields_ = [
        ("iterations", ct.c_size_t),
        ("h_applies", ct.c_size_t),
        ("converged", ct.c_int),
        ("max_residual", ct.c_double),
    ]


PROFILE_FIELDS = (
    "apply_h_ns",
    "apply_local_ns",
    "apply_nonlocal_ns",
    "density_ns",
    "subspace_ns",
    "apply_h_calls",
    "apply_h_columns",
    "local_plane_inv_ns",
    "local_xline_ns",
    "local_plane_fwd_ns",
    "local_plane_inv_launches",
    "local_xline_launches",
    "local_plane_fwd_launches",
    "nl_project_ns",
    "nl_dij_ns",
    "nl_backproject_ns",
    "kernel_launches",
    "local_layout",
)


class _TuneReport(ct.Structure):
    _fields_ = [("fft_path", ct.c_int), ("box_budget_mb", ct.c_double), ("proj_splits", ct.c_int), ("back_splits", ct.c_int),
                ("default_ms", ct.c_double), ("tuned_ms", ct.c_double), ("candidates", ct.c_int)]


class _Profile(ct.Structure):
    _fields_ = [(f, ct.c_uint64) for f in PROFILE_FIELDS]


class _HxcTerms(ct.Structure):
    _fields_ = [("e_hartree", ct.c_double), ("e_xc", ct.c_double), ("int_vin_rho", ct.c_double)]


_lib = None


def load_library(path: str = LIB_PATH) -> ct.CDLL:
    """Load libdftcuda.so; raises when it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libdftcuda.so not built at {path}; run __graft_entry__.build()")
    lib = ct.CDLL(path)
    vp, sz, dp, ip = ct.c_void_p, ct.c_size_t, ct.c_void_p, ct.c_int
    lib.dftcuda_status_string.restype = ct.c_char_p
    lib.dftcuda_status_string.argtypes = [ip]
    lib.dftcuda_last_error_message.restype = ct.c_char_p
    lib.dftcuda_device_count.restype = ip
    lib.dftcuda_kctx_create.argtypes = [ct.POINTER(vp), ip, ip, ip, ct.c_double, sz, vp, vp, vp, ip]
    lib.dftcuda_kctx_destroy.argtypes = [vp]
    lib.dftcuda_kctx_npw.argtypes = [vp]
    lib.dftcuda_kctx_npw.restype = sz
    lib.dftcuda_set_vloc.argtypes = [vp, dp]
    lib.dftcuda_set_projectors.argtypes = [vp, sz, ct.POINTER(_Species), sz, vp, vp]
    lib.dftcuda_apply_h_batch.argtypes = [vp, dp, dp, sz, sz]
    lib.dftcuda_apply_h.argtypes = [vp, dp, dp, sz]
    lib.dftcuda_apply_h_batch_async.argtypes = [vp, dp, dp, sz, vp]
    lib.dftcuda_nonlocal_energies.argtypes = [vp, dp, sz, sz, dp]
    lib.dftcuda_eig_solve.argtypes = [vp, dp, sz, ct.POINTER(_EigOpts), dp, sz, dp, dp, ct.POINTER(_EigInfo)]
    lib.dftcuda_accumulate_density.argtypes = [vp, dp, sz, sz, dp, dp]
    lib.dftcuda_fft_plan_create.argtypes = [ct.POINTER(vp), ip, ip, ip]
    lib.dftcuda_fft_plan_destroy.argtypes = [vp]
    lib.dftcuda_fft3d.argtypes = [vp, dp, ip]
    lib.dftcuda_kctx_set_profiling.argtypes = [vp, ip]
    lib.dftcuda_kctx_get_profile.argtypes = [vp, ct.POINTER(_Profile)]
    lib.dftcuda_accumulate_density_noalloc.argtypes = [vp, dp, sz, sz, dp, dp]
    lib.dftcuda_hermitian_eigen_decomp.argtypes = [sz, dp, sz, dp, dp]
    pp = ct.POINTER(ct.c_void_p)
    lib.dftcuda_kctx_autotune.argtypes = [vp, sz, ct.POINTER(_TuneReport)]
    lib.dftcuda_kctx_set_preconditioner.argtypes = [vp, ip, vp, sz]
    lib.dftcuda_precond_mlp_loss_grad.argtypes = [sz, sz, vp, vp, vp, vp, vp, vp, dp, vp]
    lib.dftcuda_precond_mlp_train.argtypes = [sz, sz, vp, vp, vp, vp, vp, vp, sz, ct.c_float, dp]
    lib.dftcuda_fno_forward.argtypes = [ip, ip, ip, vp, vp, vp]
    lib.dftcuda_fno_loss_grad.argtypes = [sz, vp, vp, vp, vp, vp, dp, vp]
    lib.dftcuda_fno_train.argtypes = [sz, vp, vp, vp, vp, vp, sz, ct.c_float, dp]
    lib.dftcuda_eig_solve_batch.argtypes = [sz, pp, pp, sz, ct.POINTER(_EigOpts), pp, ct.POINTER(ct.c_size_t), pp, pp, ct.POINTER(_EigInfo)]
    lib.dftcuda_pctx_create.argtypes = [ct.POINTER(vp), ip, ip, ip, ct.c_double, vp, ip]
    lib.dftcuda_pctx_destroy.argtypes = [vp]
    lib.dftcuda_hxc_potential.argtypes = [vp, dp, dp, dp, ct.POINTER(_HxcTerms)]
    lib.dftcuda_potential_real.argtypes = [vp, dp, dp, dp]
    lib.dftcuda_pulay_mix.argtypes = [vp, dp, dp, sz, ct.c_double]
    lib.dftcuda_pulay_reset.argtypes = [vp]
    lib.dftcuda_ionic_potential.argtypes = [vp, ip, vp, ip, vp, vp, ct.c_double, dp, dp]
    lib.dftcuda_pctx_set_functional.argtypes = [vp, ip]
    lib.dftcuda_local_forces.argtypes = [vp, ip, vp, ip, vp, vp, ct.c_double, dp, dp]
    lib.dftcuda_nonlocal_forces.argtypes = [vp, dp, sz, sz, dp, dp]
    lib.dftcuda_radial_table.argtypes = [ip, sz, dp, dp, dp, sz, ct.c_double, dp]
    lib.dftcuda_plane_wave_basis.argtypes = [dp, ct.c_double, dp, sz, vp, dp, dp, dp, ct.POINTER(ct.c_size_t)]
    lib.dftcuda_projector_phi.argtypes = [ip, sz, ct.c_double, dp, sz, dp, dp]
    lib.dftcuda_symmetrize_density.argtypes = [vp, ip, vp, vp, vp]
    lb = ct.c_long
    lib.dftcuda_complex_gemm.argtypes = [ip, sz, sz, sz, vp, lb, ip, ip, vp, lb, ip, ip, vp, lb, lb, ct.c_double, ct.c_double]
    lib.dftcuda_debug_set_wait_limits.argtypes = [lb, ip]
    lib.dftcuda_debug_fail_alloc.argtypes = [lb]
    lib.dftcuda_fermi_occupations.argtypes = [sz, sz, dp, dp, ct.c_double, ct.c_double, ct.c_double, dp, dp, dp]
    lib.dftcuda_nonlocal_stress.argtypes = [vp, dp, sz, ct.POINTER(ct.c_void_p), dp, sz, sz, dp, dp]
    lib.dftcuda_ionic_potential_radial.argtypes = [vp, ip, vp, vp, vp, vp, vp, ip, vp, vp, ct.c_double, dp, dp]
    lib.dftcuda_local_forces_radial.argtypes = [vp, ip, vp, vp, vp, vp, vp, ip, vp, vp, ct.c_double, dp, dp]
    _lib = lib
    return lib


def _check(status: int):
    if status == 0:
        return
    lib = load_library()
    msg = lib.dftcuda_last_error_message().decode(errors="replace")
    cls = _ERRORS.get(status, DftCudaError)
    raise cls(f"{lib.dftcuda_status_string(status).decode()}: {msg}")


def _require_device():
    if load_library().dftcuda_device_count() < 1:
        raise CudaError("no CUDA device visible to libdftcuda")


def _ptr(a):
    """Raw pointer of a numpy array (host) or a torch tensor (host or CUDA)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


@dataclass
class Options:
    """lobpcg/common.zig:44-52."""

    max_iter: int = 40
    tol: float = 1e-6
    max_subspace: int = 0
    block_size: int = 0
    init_diagonal: bool = False
    init_vectors: Optional[np.ndarray] = None
    init_vectors_cols: int = 0


@dataclass
class EigenDecomp:
    """linalg.zig:69-79 plus the solver's run statistics."""

    values: np.ndarray
    vectors: np.ndarray  # (nbands, n)
    n: int
    iterations: int = 0
    h_applies: int = 0
    converged: bool = True
    max_residual: float = 0.0


@dataclass
class SpeciesProjectors:
    """A NonlocalSpecies (scf/nonlocal_context.zig:9-41): l per radial projector, radial D_ij (Ry)
    and phi[m_total, n_pw] = 4 pi R(|k+G|) Y_lm(k+G)."""

    l_list: list
    dij: np.ndarray
    phi: np.ndarray


class KpointContext:
    """One k-point's H|psi> operator on the GPU (ApplyContext + KpointApplyCache of apply.zig:45-169)."""

    def __init__(self, nx, ny, nz, volume, hkl, kinetic, gcart, precision=PRECISION_FP64):
        lib = load_library()
        _require_device()
        self._lib = lib
        self.hkl = np.ascontiguousarray(hkl, dtype=np.int32)
        self.kinetic = np.ascontiguousarray(kinetic, dtype=np.float64)
        self.gcart = np.ascontiguousarray(gcart, dtype=np.float64)
        self.n = int(self.kinetic.size)
        self.dims = (int(nx), int(ny), int(nz))
        self.volume = float(volume)
        self.precision = precision
        h = ct.c_void_p()
        _check(lib.dftcuda_kctx_create(ct.byref(h), nx, ny, nz, float(volume), self.n, _ptr(self.hkl), _ptr(self.kinetic), _ptr(self.gcart), precision))
        self._h = h

    @classmethod
    def from_basis(cls, grid_dims, volume, basis, precision=PRECISION_FP64):
        return cls(grid_dims[0], grid_dims[1], grid_dims[2], volume, basis.hkl, basis.kinetic, basis.cart, precision)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.dftcuda_kctx_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_vloc(self, local_r):
        a = local_r if hasattr(local_r, "data_ptr") else np.ascontiguousarray(local_r, dtype=np.float64)
        _check(self._lib.dftcuda_set_vloc(self._h, _ptr(a)))

    def set_projectors(self, species, atom_species, atom_pos):
        """species: list[SpeciesProjectors]; atom_species[natom] index; atom_pos[natom,3] Cartesian bohr."""
        keep = []
        arr = (_Species * max(len(species), 1))()
        for i, sp in enumerate(species):
            l = np.ascontiguousarray(sp.l_list, dtype=np.int32)
            d = np.ascontiguousarray(sp.dij, dtype=np.float64)
            phi = np.ascontiguousarray(sp.phi, dtype=np.float64)
            keep += [l, d, phi]
            arr[i].beta_count = l.size
            arr[i].l_list = l.ctypes.data_as(ct.POINTER(ct.c_int32))
            arr[i].dij = d.ctypes.data_as(ct.POINTER(ct.c_double))
            arr[i].m_total = phi.shape[0] if phi.ndim == 2 else 0
            arr[i].phi = phi.ctypes.data_as(ct.POINTER(ct.c_double))
        asp = np.ascontiguousarray(atom_species, dtype=np.int32)
        apos = np.ascontiguousarray(atom_pos, dtype=np.float64)
        _check(self._lib.dftcuda_set_projectors(self._h, len(species), arr, asp.size, _ptr(asp), _ptr(apos)))

    # Operator.apply / apply_batch -------------------------------------------------------------
    def apply_hamiltonian_batched(self, x_batch, y_batch=None, n=None, ncols=None):
        if isinstance(x_batch, np.ndarray):
            x_batch = np.ascontiguousarray(x_batch, dtype=np.complex128)
            ncols = x_batch.size // self.n if ncols is None else ncols
            if y_batch is None:
                y_batch = np.empty_like(x_batch)
        n = self.n if n is None else n
        if ncols is None:
            ncols = x_batch.numel() // self.n
        _check(self._lib.dftcuda_apply_h_batch(self._h, _ptr(x_batch), _ptr(y_batch), n, ncols))
        return y_batch

    def apply_hamiltonian(self, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty_like(x) if y is None else y
        _check(self._lib.dftcuda_apply_h(self._h, _ptr(x), _ptr(y), x.size))
        return y

    def apply_hamiltonian_async(self, x_dev, y_dev, ncols, stream=None):
        """Device tensors only, no host synchronisation (the device-resident bench path)."""
        _check(self._lib.dftcuda_apply_h_batch_async(self._h, _ptr(x_dev), _ptr(y_dev), ncols, stream))

    def set_profiling(self, enable: bool = True):
        """Start (and clear) or stop the device-time ScfProfile counters of this context."""
        _check(self._lib.dftcuda_kctx_set_profiling(self._h, 1 if enable else 0))

    def profile(self) -> dict:
        p = _Profile()
        _check(self._lib.dftcuda_kctx_get_profile(self._h, ct.byref(p)))
        return {f: int(getattr(p, f)) for f in PROFILE_FIELDS}

    def nonlocal_energies(self, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128).reshape(-1, self.n)
        e = np.empty(psi.shape[0])
        _check(self._lib.dftcuda_nonlocal_energies(self._h, _ptr(psi), self.n, psi.shape[0], _ptr(e)))
        return e

    def accumulate_band_density(self, vectors, weights, rho):
        """rho (N, FFT order x fastest) += sum_b weights_b |psi_b(r)|^2 / Omega."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if isinstance(vectors, np.ndarray):
            vectors = np.ascontiguousarray(vectors, dtype=np.complex128).reshape(-1, self.n)
        _check(self._lib.dftcuda_accumulate_density(self._h, _ptr(vectors), self.n, w.size, _ptr(w), _ptr(rho)))
        return rho

    def nonlocal_forces(self, vectors, weights, natoms: int) -> np.ndarray:
        """Nonlocal Hellmann-Feynman forces (natoms, 3) in Ry/bohr of the bands `vectors` (nbands, n)
        with weights k weight x occupation x spin, for the atoms given to set_projectors."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if isinstance(vectors, np.ndarray):
            vectors = np.ascontiguousarray(vectors, dtype=np.complex128).reshape(-1, self.n)
        out = np.zeros((natoms, 3))
        _check(self._lib.dftcuda_nonlocal_forces(self._h, _ptr(vectors), self.n, w.size, w.ctypes.data, out.ctypes.data))
        return out

    def nonlocal_stress(self, kpg, dphi, vectors, weights) -> np.ndarray:
        """Nonlocal stress (3, 3) in Ry/bohr^3 of the bands (nbands, n) with weights f_n, a <= b filled
        (dftcuda_nonlocal_stress).  kpg (n, 3) = k + G; dphi: per species (m_total, 3, n) derivative
        projectors (system.projector_derivatives)."""
        q = np.ascontiguousarray(kpg, dtype=np.float64).reshape(self.n, 3)
        tabs = [np.ascontiguousarray(np.transpose(np.asarray(d, dtype=np.float64), (1, 0, 2))) for d in dphi]
        arr = (ct.c_void_p * max(len(tabs), 1))(*[t.ctypes.data for t in tabs])
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if isinstance(vectors, np.ndarray):
            vectors = np.ascontiguousarray(vectors, dtype=np.complex128).reshape(-1, self.n)
        out = np.zeros(9)
        _check(self._lib.dftcuda_nonlocal_stress(self._h, q.ctypes.data, len(tabs), arr, _ptr(vectors), self.n, w.size, w.ctypes.data,
                                                 out.ctypes.data))
        return out.reshape(3, 3)

    def accumulate_band_density_noalloc(self, vectors_dev, weights_dev, rho_dev, nbands=None):
        """Same result as accumulate_band_density for device tensors, without any device allocation
        (for callers that cannot allocate: the library uses a fixed 48 MiB scratch array in its
        device image instead).  Calls that overlap on the GPU share that array and race."""
        nb = weights_dev.numel() if nbands is None else nbands
        _check(self._lib.dftcuda_accumulate_density_noalloc(self._h, _ptr(vectors_dev), self.n, nb, _ptr(weights_dev), _ptr(rho_dev)))
        return rho_dev

    def set_preconditioner(self, kind: int, params=None):
        """Preconditioner of this context's Davidson correction step (PRECOND_*); the learned one
        takes its PRECOND_MLP_PARAMS float32 weights."""
        buf = None
        n = 0
        if params is not None:
            buf = np.ascontiguousarray(params, dtype=np.float32)
            n = buf.size
        _check(self._lib.dftcuda_kctx_set_preconditioner(self._h, kind, _ptr(buf), n))

    def autotune(self, ncols: int) -> dict:
        """Time candidate H|psi> launch configurations on ncols columns and keep the fastest."""
        r = _TuneReport()
        _check(self._lib.dftcuda_kctx_autotune(self._h, ncols, ct.byref(r)))
        return {f: getattr(r, f) for f, _ in r._fields_}

    def hermitian_eigen_decomp_iterative(self, diag, nbands, opts: Options = Options()) -> EigenDecomp:
        """iterative.zig:67-76 -> lobpcg_serial.solve with this context as the Operator."""
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        if diag.size != self.n:
            raise InvalidMatrixSize("diag length != n")
        o = _EigOpts(opts.max_iter, opts.tol, opts.max_subspace, opts.block_size, 1 if opts.init_diagonal else 0)
        init = None
        icols = 0
        if opts.init_vectors is not None:
            init = np.ascontiguousarray(opts.init_vectors, dtype=np.complex128).reshape(-1, self.n)
            icols = opts.init_vectors_cols or init.shape[0]
        vals = np.empty(nbands)
        vecs = np.empty((nbands, self.n), dtype=np.complex128)
        info = _EigInfo()
        _check(self._lib.dftcuda_eig_solve(self._h, _ptr(diag), nbands, ct.byref(o), _ptr(init), icols, _ptr(vals), _ptr(vecs), ct.byref(info)))
        return EigenDecomp(vals, vecs, self.n, info.iterations, info.h_applies, bool(info.converged), info.max_residual)


def hermitian_eigen_decomp_iterative_batch(ctxs, diags, nbands, opts: Options = Options(), init_vectors=None,
                                           device: bool = False) -> list:
    """The iterative solver for several k-point contexts at once (dftcuda_eig_solve_batch): the runs
    advance in lockstep on their contexts' streams.  init_vectors: None or a list with an (icols, n_k)
    array (numpy, or a CUDA complex128 tensor read in place) or None per context.  device=True
    returns the eigenvectors as CUDA tensors (nothing crosses to the host but the eigenvalues).
    Returns one EigenDecomp per context."""
    lib = load_library()
    nk = len(ctxs)
    if nk == 0:
        return []
    o = _EigOpts(opts.max_iter, opts.tol, opts.max_subspace, opts.block_size, 1 if opts.init_diagonal else 0)
    keep = []
    d_arr = (ct.c_void_p * nk)()
    i_arr = (ct.c_void_p * nk)()
    ic_arr = (ct.c_size_t * nk)()
    v_arr = (ct.c_void_p * nk)()
    x_arr = (ct.c_void_p * nk)()
    out = []
    for i, kc in enumerate(ctxs):
        d = np.ascontiguousarray(diags[i], dtype=np.float64)
        if d.size != kc.n:
            raise InvalidMatrixSize("diag length != n")
        keep.append(d)
        d_arr[i] = d.ctypes.data
        if init_vectors is not None and init_vectors[i] is not None:
            iv = init_vectors[i]
            if _is_torch_cuda(iv):
                import torch

                if iv.dtype != torch.complex128 or not iv.is_contiguous() or iv.numel() % kc.n:
                    raise InvalidMatrixSize("init_vectors: contiguous complex128 tensors of whole columns")
                i_arr[i] = iv.data_ptr()
                ic_arr[i] = iv.numel() // kc.n
            else:
                iv = np.ascontiguousarray(iv, dtype=np.complex128).reshape(-1, kc.n)
                i_arr[i] = iv.ctypes.data
                ic_arr[i] = iv.shape[0]
            keep.append(iv)
        vals = np.empty(nbands)
        if device:
            import torch

            vecs = torch.empty((nbands, kc.n), dtype=torch.complex128, device="cuda")
        else:
            vecs = np.empty((nbands, kc.n), dtype=np.complex128)
        out.append((vals, vecs))
        v_arr[i] = vals.ctypes.data
        x_arr[i] = _ptr(vecs)
    h_arr = (ct.c_void_p * nk)(*[kc.handle.value for kc in ctxs])
    infos = (_EigInfo * nk)()
    _check(lib.dftcuda_eig_solve_batch(nk, h_arr, d_arr, nbands, ct.byref(o), i_arr, ic_arr, v_arr, x_arr, infos))
    return [EigenDecomp(v, x, kc.n, inf.iterations, inf.h_applies, bool(inf.converged), inf.max_residual)
            for (v, x), kc, inf in zip(out, ctxs, infos)]


def _mlp_arrays(off, feat, cc, w, dnorm):
    off = np.ascontiguousarray(off, dtype=np.int32)
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    cc = np.ascontiguousarray(np.stack([np.real(cc), np.imag(cc)], axis=1), dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    dnorm = np.ascontiguousarray(dnorm, dtype=np.float32)
    return off, feat, cc, w, dnorm


def precond_mlp_loss_grad(params, off, feat, cc, w, dnorm):
    """Loss and gradient of the learned preconditioner on the GPU (dftcuda_precond_mlp_loss_grad)."""
    lib = load_library()
    _require_device()
    off, feat, cc, w, dnorm = _mlp_arrays(off, feat, cc, w, dnorm)
    p = np.ascontiguousarray(params, dtype=np.float32)
    loss = ct.c_double(0.0)
    grad = np.zeros(PRECOND_MLP_PARAMS, dtype=np.float32)
    _check(lib.dftcuda_precond_mlp_loss_grad(len(off) - 1, feat.shape[0], _ptr(off), _ptr(feat), _ptr(cc), _ptr(w), _ptr(dnorm),
                                             _ptr(p), ct.addressof(loss), _ptr(grad)))
    return loss.value, grad


def precond_mlp_train(params, off, feat, cc, w, dnorm, steps: int, lr: float = 1e-3):
    """`steps` full-batch Adam steps on the GPU (dftcuda_precond_mlp_train); returns the trained
    parameters and the loss before each step."""
    lib = load_library()
    _require_device()
    off, feat, cc, w, dnorm = _mlp_arrays(off, feat, cc, w, dnorm)
    p = np.array(params, dtype=np.float32)
    hist = np.zeros(steps, dtype=np.float64)
    _check(lib.dftcuda_precond_mlp_train(len(off) - 1, feat.shape[0], _ptr(off), _ptr(feat), _ptr(cc), _ptr(w), _ptr(dnorm),
                                         _ptr(p), steps, lr, _ptr(hist)))
    return p, hist


def _fno_set(samples):
    """samples: list of (dims (nx, ny, nz), u [2][N], target [N] or None)."""
    dims = np.ascontiguousarray([d for dd, _, _ in samples for d in dd], dtype=np.int32)
    sizes = [int(np.prod(dd)) for dd, _, _ in samples]
    offs = np.ascontiguousarray(np.concatenate([[0], np.cumsum(sizes)]), dtype=np.uint64)
    u = np.ascontiguousarray(np.concatenate([np.asarray(uu, np.float32).reshape(-1) for _, uu, _ in samples]), dtype=np.float32)
    t = None
    if all(tt is not None for _, _, tt in samples):
        t = np.ascontiguousarray(np.concatenate([np.asarray(tt, np.float32).reshape(-1) for _, _, tt in samples]), dtype=np.float32)
    return dims, offs, u, t


def fno_forward(params, u, dims):
    """The learned first-density operator on one cell: u [2][nx ny nz] -> [nx ny nz] (float32)."""
    lib = load_library()
    _require_device()
    nx, ny, nz = dims
    uu = np.ascontiguousarray(u, dtype=np.float32).reshape(-1)
    p = np.ascontiguousarray(params, dtype=np.float32)
    out = np.empty(nx * ny * nz, dtype=np.float32)
    _check(lib.dftcuda_fno_forward(nx, ny, nz, _ptr(uu), _ptr(p), _ptr(out)))
    return out


def fno_loss_grad(params, samples):
    lib = load_library()
    _require_device()
    dims, offs, u, t = _fno_set(samples)
    p = np.ascontiguousarray(params, dtype=np.float32)
    loss = ct.c_double(0.0)
    grad = np.zeros(FNO_PARAMS, dtype=np.float32)
    _check(lib.dftcuda_fno_loss_grad(len(samples), _ptr(dims), _ptr(offs), _ptr(u), _ptr(t), _ptr(p), ct.addressof(loss), _ptr(grad)))
    return loss.value, grad


def fno_train(params, samples, steps: int, lr: float = 1e-3):
    """`steps` full-batch Adam steps on the GPU (dftcuda_fno_train); returns (params, loss history)."""
    lib = load_library()
    _require_device()
    dims, offs, u, t = _fno_set(samples)
    p = np.array(params, dtype=np.float32)
    hist = np.zeros(steps, dtype=np.float64)
    _check(lib.dftcuda_fno_train(len(samples), _ptr(dims), _ptr(offs), _ptr(u), _ptr(t), _ptr(p), steps, lr, _ptr(hist)))
    return p, hist


class PotentialContext:
    """SCF potential build and Pulay mixing on the device (dftcuda_pctx_*): the FFT box `dims`
    (nx, ny, nz; x fastest), the cell volume, the reciprocal vectors (rows b1, b2, b3) and the Pulay
    history length.  Arrays may be numpy (host) or CUDA torch tensors; results come back in the
    kind given (numpy in -> numpy out)."""

    FUNCTIONALS = {"lda": 0, "pbe": 1}

    def __init__(self, dims, volume: float, recip, history: int = 8, functional: str = "lda"):
        lib = load_library()
        _require_device()
        self.dims = tuple(int(d) for d in dims)
        self.N = self.dims[0] * self.dims[1] * self.dims[2]
        r = np.ascontiguousarray(np.asarray(recip, dtype=np.float64).reshape(3, 3))
        h = ct.c_void_p()
        _check(lib.dftcuda_pctx_create(ct.byref(h), *self.dims, float(volume), r.ctypes.data, int(history)))
        self._h = h
        if functional not in self.FUNCTIONALS:
            raise InvalidArgument(f"functional must be one of {sorted(self.FUNCTIONALS)}")
        _check(lib.dftcuda_pctx_set_functional(self._h, self.FUNCTIONALS[functional]))

    def _out_like(self, ref, shape, dtype):
        if _is_torch_cuda(ref):
            import torch

            return torch.empty(shape, dtype={np.complex128: torch.complex128, np.float64: torch.float64}[dtype], device=ref.device)
        return np.empty(shape, dtype=dtype)

    def hxc(self, rho, v_in=None, out=None):
        """(V_H + V_xc)(G) of rho(r) and the energy terms {e_hartree, e_xc, int_vin_rho}."""
        rho = _as_array(rho, np.float64, self.N)
        v_in = None if v_in is None else _as_array(v_in, np.complex128, self.N)
        if out is None:
            out = self._out_like(rho, (self.N,), np.complex128)
        t = _HxcTerms()
        _check(load_library().dftcuda_hxc_potential(self._h, _ptr(rho), _ptr(v_in) if v_in is not None else None, _ptr(out), ct.byref(t)))
        return out, {"e_hartree": t.e_hartree, "e_xc": t.e_xc, "int_vin_rho": t.int_vin_rho}

    def real(self, v_g, vloc=None, out=None):
        """V(r) = vloc(r) + FFT^-1 v(G) (the local potential for set_vloc)."""
        v_g = _as_array(v_g, np.complex128, self.N)
        vloc = None if vloc is None else _as_array(vloc, np.float64, self.N)
        if out is None:
            out = self._out_like(v_g, (self.N,), np.float64)
        _check(load_library().dftcuda_potential_real(self._h, _ptr(v_g), _ptr(vloc) if vloc is not None else None, _ptr(out)))
        return out

    def symmetrize(self, rho, ops):
        """Density symmetrisation in place (dftcuda_symmetrize_density): ops is a list of
        (rot, k_rot, trans) or of (k_rot, trans), k_rot acting on Miller indices, trans fractional."""
        rho = _as_array(rho, np.float64, self.N)
        kr = np.ascontiguousarray([np.asarray(o[-2], dtype=np.int32).reshape(9) for o in ops], dtype=np.int32).reshape(-1)
        tr = np.ascontiguousarray([np.asarray(o[-1], dtype=np.float64).reshape(3) for o in ops], dtype=np.float64).reshape(-1)
        _check(load_library().dftcuda_symmetrize_density(self._h, len(ops), kr.ctypes.data if kr.size else None,
                                                         tr.ctypes.data if tr.size else None, _ptr(rho)))
        return rho

    def pulay_mix(self, x, residual, beta: float):
        """Pulay step in place on x (float64, any length; complex arrays as their interleaved view)."""
        n = _nbytes(x) // 8
        if _nbytes(residual) != _nbytes(x):
            raise InvalidMatrixSize("pulay_mix: x and residual differ in size")
        _check(load_library().dftcuda_pulay_mix(self._h, _ptr(x), _ptr(residual), n, float(beta)))
        return x

    def reset(self):
        _check(load_library().dftcuda_pulay_reset(self._h))

    def local_forces(self, gth, atom_species, positions, rho, g2max: float = 0.0) -> np.ndarray:
        """Local-pseudopotential forces (natoms, 3) in Ry/bohr from the density rho (numpy or CUDA)."""
        g = np.ascontiguousarray(np.asarray(gth, dtype=np.float64).reshape(-1, 6))
        sp = np.ascontiguousarray(atom_species, dtype=np.int32)
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        rho = _as_array(rho, np.float64, self.N)
        out = np.empty((sp.size, 3))
        _check(load_library().dftcuda_local_forces(self._h, g.shape[0], g.ctypes.data, sp.size, sp.ctypes.data, pos.ctypes.data,
                                                   float(g2max), _ptr(rho), out.ctypes.data))
        return out

    def ionic(self, gth, atom_species, positions, g2max: float = 0.0, device: bool = False):
        """V_loc(r) of GTH-local pseudopotentials: gth (nspecies, 6) = Z, r_loc, C1..C4; atoms by
        species index and Cartesian bohr positions.  Returns (V(G), V_loc(r)), numpy or CUDA tensors."""
        g = np.ascontiguousarray(np.asarray(gth, dtype=np.float64).reshape(-1, 6))
        sp = np.ascontiguousarray(atom_species, dtype=np.int32)
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        if device:
            import torch

            vg = torch.empty(self.N, dtype=torch.complex128, device="cuda")
            vr = torch.empty(self.N, dtype=torch.float64, device="cuda")
        else:
            vg = np.empty(self.N, dtype=np.complex128)
            vr = np.empty(self.N, dtype=np.float64)
        _check(load_library().dftcuda_ionic_potential(self._h, g.shape[0], g.ctypes.data, sp.size, sp.ctypes.data, pos.ctypes.data,
                                                      float(g2max), _ptr(vg), _ptr(vr)))
        return vg, vr

    def ionic_radial(self, meshes, atom_species, positions, g2max: float = 0.0, device: bool = False):
        """V_loc from each species' radial mesh with the reference's short-range form factor
        (dftcuda_ionic_potential_radial): meshes [(r, rab, vloc_Ry, z_valence)] per species.
        Returns (V(G), V_loc(r)), numpy or CUDA tensors."""
        off, r, rab, vl, z = _radial_meshes(meshes)
        sp = np.ascontiguousarray(atom_species, dtype=np.int32)
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        if device:
            import torch

            vg = torch.empty(self.N, dtype=torch.complex128, device="cuda")
            vr = torch.empty(self.N, dtype=torch.float64, device="cuda")
        else:
            vg = np.empty(self.N, dtype=np.complex128)
            vr = np.empty(self.N, dtype=np.float64)
        _check(load_library().dftcuda_ionic_potential_radial(self._h, len(meshes), off.ctypes.data, r.ctypes.data, rab.ctypes.data,
                                                             vl.ctypes.data, z.ctypes.data, sp.size, sp.ctypes.data, pos.ctypes.data,
                                                             float(g2max), _ptr(vg), _ptr(vr)))
        return vg, vr

    def local_forces_radial(self, meshes, atom_species, positions, rho, g2max: float = 0.0) -> np.ndarray:
        """Local-pseudopotential forces (natoms, 3) in Ry/bohr from each species' radial mesh."""
        off, r, rab, vl, z = _radial_meshes(meshes)
        sp = np.ascontiguousarray(atom_species, dtype=np.int32)
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        rho = _as_array(rho, np.float64, self.N)
        out = np.empty((sp.size, 3))
        _check(load_library().dftcuda_local_forces_radial(self._h, len(meshes), off.ctypes.data, r.ctypes.data, rab.ctypes.data,
                                                          vl.ctypes.data, z.ctypes.data, sp.size, sp.ctypes.data, pos.ctypes.data,
                                                          float(g2max), _ptr(rho), out.ctypes.data))
        return out

    def close(self):
        if self._h:
            load_library().dftcuda_pctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fermi_occupations(values, kweights, nelec: float, sigma: float, spin: float = 2.0):
    """Fermi level, Fermi-Dirac occupations and energy sums of an eigenvalue table on the device
    (dftcuda_fermi_occupations; find_fermi_level_spin, fermi_level.zig:61-124).  values (nk, nbands),
    kweights (nk,).  Returns (mu, occ (nk, nbands), band_sum, entropy_sum) with band_sum =
    sum spin w_k f e and entropy_sum = sum spin w_k S(f)."""
    lib = load_library()
    _require_device()
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.ndim != 2:
        raise InvalidMatrixSize("values must be (nk, nbands)")
    w = np.ascontiguousarray(kweights, dtype=np.float64)
    if w.size != v.shape[0]:
        raise InvalidMatrixSize("one weight per k-point")
    mu = ct.c_double(0.0)
    occ = np.zeros_like(v)
    sums = np.zeros(2)
    _check(lib.dftcuda_fermi_occupations(v.shape[0], v.shape[1], v.ctypes.data, w.ctypes.data, float(nelec), float(sigma),
                                         float(spin), ct.addressof(mu), occ.ctypes.data, sums.ctypes.data))
    return mu.value, occ, float(sums[0]), float(sums[1])


def _radial_meshes(meshes):
    """Packs [(r, rab, vloc, z)] per species into (offsets, r, rab, vloc, z) for the *_radial calls."""
    off = np.zeros(len(meshes) + 1, dtype=np.uint64)
    for i, (r, _, _, _) in enumerate(meshes):
        off[i + 1] = off[i] + len(r)
    cat = [np.ascontiguousarray(np.concatenate([np.asarray(m[j], dtype=np.float64) for m in meshes])) for j in range(3)]
    z = np.ascontiguousarray([float(m[3]) for m in meshes], dtype=np.float64)
    return off, cat[0], cat[1], cat[2], z


def debug_set_wait_limits(polls: int = 0, unreachable: bool = False):
    """Failure injection for the bounded device waits (dftcuda_debug_set_wait_limits): polls > 0 sets
    the subspace eigensolver's grid-barrier poll budget, unreachable makes every barrier wait run it
    out (the call then raises Timeout).  debug_set_wait_limits() restores the defaults."""
    _check(load_library().dftcuda_debug_set_wait_limits(int(polls), 1 if unreachable else 0))


def debug_fail_alloc(after: int = -1):
    """Failure injection for the out-of-memory path (dftcuda_debug_fail_alloc): after >= 0 makes the
    after-th following device allocation of the library fail once (the call that makes it raises
    OutOfMemory); debug_fail_alloc() cancels a planned failure."""
    _check(load_library().dftcuda_debug_fail_alloc(int(after)))


def _is_torch_cuda(a) -> bool:
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


def _as_array(a, dtype, n):
    """A contiguous array of n elements of dtype: CUDA tensors are checked, numpy data converted."""
    if _is_torch_cuda(a):
        import torch

        want = {np.complex128: torch.complex128, np.float64: torch.float64}[dtype]
        if a.dtype != want or a.numel() != n or not a.is_contiguous():
            raise InvalidMatrixSize(f"expected a contiguous CUDA tensor of {n} {want}")
        return a
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.size != n:
        raise InvalidMatrixSize(f"expected {n} elements, got {a.size}")
    return a


def _nbytes(a) -> int:
    if _is_torch_cuda(a):
        return a.numel() * a.element_size()
    return np.asarray(a).nbytes


def radial_table(l: int, r, rbeta, rab, gmax: float, npts: int = 2048):
    """Radial projector table of one beta on the device (dftcuda_radial_table): values on
    q_i = i gmax / (npts - 1).  Returns (values, gmax, dq) like system.radial_table."""
    lib = load_library()
    _require_device()
    r = np.ascontiguousarray(r, dtype=np.float64)
    rbeta = np.ascontiguousarray(rbeta, dtype=np.float64)
    rab = np.ascontiguousarray(rab, dtype=np.float64)
    out = np.empty(int(npts))
    _check(lib.dftcuda_radial_table(int(l), r.size, r.ctypes.data, rbeta.ctypes.data, rab.ctypes.data, out.size, float(gmax), out.ctypes.data))
    return out, float(gmax), float(gmax) / (npts - 1)


def plane_wave_basis(recip, ecut: float, k_cart):
    """The plane-wave basis of one k-point built on the device (dftcuda_plane_wave_basis): returns
    (hkl int32 [n][3], gcart [n][3], kpg [n][3], kinetic [n]) in the reference's order."""
    lib = load_library()
    _require_device()
    recip = np.ascontiguousarray(recip, dtype=np.float64).reshape(9)
    k = np.ascontiguousarray(k_cart, dtype=np.float64).reshape(3)
    n = ct.c_size_t(0)
    _check(lib.dftcuda_plane_wave_basis(recip.ctypes.data, float(ecut), k.ctypes.data, 0, None, None, None, None, ct.byref(n)))
    m = int(n.value)
    hkl = np.empty((m, 3), dtype=np.int32)
    g = np.empty((m, 3))
    q = np.empty((m, 3))
    kin = np.empty(m)
    _check(lib.dftcuda_plane_wave_basis(recip.ctypes.data, float(ecut), k.ctypes.data, max(m, 1), hkl.ctypes.data, g.ctypes.data,
                                        q.ctypes.data, kin.ctypes.data, ct.byref(n)))
    return hkl, g, q, kin


def projector_phi(l: int, table, kpg):
    """Projector rows phi[(2l+1)][n] = 4 pi R(|k+G|) Y_lm(k+G) on the device (dftcuda_projector_phi);
    table = (values, gmax, dq) as radial_table returns."""
    lib = load_library()
    _require_device()
    vals, gmax, _ = table
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    kpg = np.ascontiguousarray(kpg, dtype=np.float64).reshape(-1, 3)
    out = np.empty((2 * int(l) + 1, kpg.shape[0]))
    _check(lib.dftcuda_projector_phi(int(l), vals.size, float(gmax), vals.ctypes.data, kpg.shape[0], kpg.ctypes.data, out.ctypes.data))
    return out


def complex_gemm(a, b, out=None, *, conj_a: bool = False, conj_b: bool = False, precision: int = 0, alpha: float = 1.0,
                 beta: float = 0.0):
    """out[r, c] = alpha * sum_k opA(a)[r, k] opB(b)[c, k] + beta * out[r, c] on the GPU
    (dftcuda_complex_gemm): a (M, K) and b (N, K) CUDA complex128 tensors, each with a unit stride
    along one of its two dimensions; opX conjugates when conj_x.  precision 0 runs the FP64 kernel,
    PRECISION_TF32 / PRECISION_TF32X3 the tensor-core kernels.  Returns out (allocated (M, N) when
    None)."""
    import torch

    lib = load_library()
    _require_device()

    def layout(t, name):
        if t.dtype != torch.complex128 or not t.is_cuda or t.dim() != 2:
            raise InvalidArgument(f"complex_gemm: {name} must be a 2-D CUDA complex128 tensor")
        sr, sk = t.stride()
        if sk == 1:
            return 1, max(sr, 1)
        if sr == 1:
            return 0, max(sk, 1)
        raise InvalidArgument(f"complex_gemm: {name} needs a unit stride along one dimension")

    M, K = a.shape
    N, K2 = b.shape
    if K2 != K:
        raise InvalidMatrixSize("complex_gemm: a and b disagree on K")
    if out is None:
        out = torch.zeros((M, N), dtype=torch.complex128, device=a.device)
    if tuple(out.shape) != (M, N) or out.dtype != torch.complex128:
        raise InvalidMatrixSize("complex_gemm: out must be (M, N) complex128")
    a_kc, lda = layout(a, "a")
    b_kc, ldb = layout(b, "b")
    torch.cuda.synchronize(a.device)
    _check(lib.dftcuda_complex_gemm(int(precision), M, N, K, a.data_ptr(), lda, a_kc, int(conj_a), b.data_ptr(), ldb, b_kc,
                                    int(conj_b), out.data_ptr(), out.stride(0), out.stride(1), float(alpha), float(beta)))
    return out


def hermitian_eigen_decomp(a, nev: Optional[int] = None) -> EigenDecomp:
    """linalg.hermitian_eigen_decomp (linalg/linalg.zig:141-151) on the GPU: the nev lowest
    eigenpairs (all when nev is None) of the Hermitian matrix a[i, j]; only its upper triangle
    (i <= j) is read, as zheev 'U' does.  vectors has shape (nev, n), one eigenvector per row."""
    lib = load_library()
    _require_device()
    a = np.asarray(a, dtype=np.complex128)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise InvalidMatrixSize("hermitian_eigen_decomp: square matrix expected")
    n = a.shape[0]
    k = n if nev is None else int(nev)
    colmajor = np.ascontiguousarray(a.T)  # memory order a[i + j n] = a[i, j]
    vals = np.empty(k, dtype=np.float64)
    vecs = np.empty((k, n), dtype=np.complex128)
    _check(lib.dftcuda_hermitian_eigen_decomp(n, _ptr(colmajor), k, _ptr(vals), _ptr(vecs)))
    return EigenDecomp(vals, vecs, n)


class Fft3dPlan:
    """Fft3dPlan with the fftw backend's semantics (fft.zig:44-263, fftw_fft.zig:141-166)."""

    def __init__(self, nx, ny, nz):
        lib = load_library()
        _require_device()
        self._lib = lib
        self.nx, self.ny, self.nz = nx, ny, nz
        h = ct.c_void_p()
        _check(lib.dftcuda_fft_plan_create(ct.byref(h), nx, ny, nz))
        self._h = h

    def forward(self, data):
        _check(self._lib.dftcuda_fft3d(self._h, _ptr(data), -1))
        return data

    def inverse(self, data):
        _check(self._lib.dftcuda_fft3d(self._h, _ptr(data), 1))
        return data

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.dftcuda_fft_plan_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
