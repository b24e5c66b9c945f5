"""The C-ABI library loads and exports every symbol include/dftcuda.h declares (no GPU needed)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "dftcuda.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(dftcuda_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree(dz):
    assert sorted(dz.ABI_SYMBOLS) == _declared()


def test_library_exports_all_symbols(dz):
    lib = dz.load_library()
    missing = [s for s in _declared() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_map_zig_errors(dz):
    lib = dz.load_library()
    names = {c: lib.dftcuda_status_string(c).decode() for c in range(-8, 1)}
    assert names[0] == "ok"
    assert names[-1] == "InvalidMatrixSize"
    assert names[-2] == "InvalidGrid"
    assert names[-3] == "LapackFailure"


def test_no_cpu_fallback_without_device(dz):
    """Without a GPU every compute entry point must fail loudly, never fall back to the CPU."""
    lib = dz.load_library()
    if lib.dftcuda_device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(dz.CudaError):
        dz.KpointContext(4, 4, 4, 1.0, np.zeros((1, 3), np.int32), np.zeros(1), np.zeros((1, 3)))
    with pytest.raises(dz.CudaError):
        dz.Fft3dPlan(4, 4, 4)


def test_null_handles_rejected(dz):
    lib = dz.load_library()
    assert lib.dftcuda_apply_h_batch(None, None, None, 0, 0) == -6
    assert lib.dftcuda_kctx_destroy(None) == 0
