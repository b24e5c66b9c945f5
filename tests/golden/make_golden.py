"""Generate the golden fixtures in this folder from the reference's own known-answer tests.

Each fixture restates the inputs of one dft-zig test and the expected output that test asserts,
computed the way that test computes it (dense loops, closed forms), together with its tolerance:

  local_potential_kat.npz  src/tests.zig:872-973  ("apply local potential vs dense", 4^3, 1e-10)
                           src/tests.zig:975-1104 ("local potential FFT vs direct", 4^3, 1e-10)
  fft_roundtrip.npz        src/features/fft/fft.zig:418-463 (6^3, 2x3x4; 1e-9),
                           src/lib/fft/fftw_fft.zig:176-227 (8^3, 24^3; 1e-9)
  bessel.json              src/tests.zig:1245-1318 (j_0..j_3 at x = 0.1 .. 20; 1e-12/1e-12/1e-10/1e-8)
  ctrap.json               src/features/math/radial_integration.zig:18-55
  lobpcg_diag.json         src/features/linalg/iterative.zig:80-203 (diag(1,2,3), diag(1,3,5,7); 1e-6)
  lcg.json                 src/features/linalg/lobpcg/common.zig:314-319 with the seed of serial.zig:111

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def local_potential_kats():
    nx = ny = nz = 4
    total = nx * ny * nz
    # test 1 (tests.zig:877-897): V(G=0)=0.5, V(1,0,0)=V(-1,0,0)=0.1 in FFT order; psi = delta(G=0)
    v1 = np.zeros(total, dtype=np.complex128)
    v1[0], v1[1], v1[nx - 1] = 0.5, 0.1, 0.1
    psi1 = np.zeros(total, dtype=np.complex128)
    psi1[0] = 1.0
    expected1 = v1.copy()  # (V psi)_G = V_G for psi = delta (tests.zig:918-924)
    # test 2 (tests.zig:980-1002): V(0)=1, V(+-1,0,0)=0.5; psi = delta(G=0); direct O(N^2) convolution
    v2 = np.zeros(total, dtype=np.complex128)
    v2[0], v2[1], v2[nx - 1] = 1.0, 0.5, 0.5
    psi2 = psi1.copy()
    direct = np.zeros(total, dtype=np.complex128)
    for gz in range(nz):
        for gy in range(ny):
            for gx in range(nx):
                g = gx + nx * (gy + ny * gz)
                s = 0.0j
                for pz in range(nz):
                    for py in range(ny):
                        for px in range(nx):
                            gp = px + nx * (py + ny * pz)
                            dq = (gx + nx - px) % nx + nx * (((gy + ny - py) % ny) + ny * ((gz + nz - pz) % nz))
                            s += v2[dq] * psi2[gp]
                direct[g] = s
    np.savez(
        os.path.join(HERE, "local_potential_kat.npz"),
        dims=np.array([nx, ny, nz]),
        v1=v1,
        psi1=psi1,
        expected1=expected1,
        v2=v2,
        psi2=psi2,
        expected2=direct,
        tol=np.array(1e-10),
    )


def fft_roundtrips():
    out = {}
    d = np.arange(216, dtype=np.float64).astype(np.complex128)  # fft.zig:424-427
    out["r6"] = d
    out["r234"] = np.arange(24, dtype=np.float64).astype(np.complex128)  # fft.zig:448-451
    out["r8"] = np.arange(512, dtype=np.float64).astype(np.complex128)  # fftw_fft.zig:186-190
    i = np.arange(24**3)
    out["r24"] = (i % 17).astype(np.float64) + 1j * (i % 13).astype(np.float64)  # fftw_fft.zig:213-216
    np.savez_compressed(
        os.path.join(HERE, "fft_roundtrip.npz"),
        dims_r6=np.array([6, 6, 6]),
        dims_r234=np.array([2, 3, 4]),
        dims_r8=np.array([8, 8, 8]),
        dims_r24=np.array([24, 24, 24]),
        tol=np.array(1e-9),
        **out,
    )


def bessel():
    xs = [0.1, 1.0, 2.0, 5.0, 10.0, 20.0]
    rows = []
    for x in xs:
        s, c = math.sin(x), math.cos(x)
        rows.append(
            {
                "x": x,
                "j0": s / x,
                "j1": s / (x * x) - c / x,
                "j2": (3.0 / (x * x) - 1.0) * s / x - 3.0 * c / (x * x),
                "j3": (15.0 / (x * x * x) - 6.0 / x) * s / x - (15.0 / (x * x) - 1.0) * c / x,
            }
        )
    doc = {"source": "src/tests.zig:1245-1318", "tol": {"j0": 1e-12, "j1": 1e-12, "j2": 1e-10, "j3": 1e-8}, "values": rows}
    with open(os.path.join(HERE, "bessel.json"), "w") as f:
        json.dump(doc, f, indent=1)


def ctrap():
    doc = {
        "source": "src/features/math/radial_integration.zig:18-55",
        "n": 20,
        "first5": [23.75 / 72.0, 95.10 / 72.0, 55.20 / 72.0, 79.30 / 72.0, 70.65 / 72.0],
        "interior_ones": [[5, 20], [10, 20], [14, 20]],
        "small_grid_ones": [[0, 5], [3, 9]],
        "x4_integral": {"n": 101, "exact": 0.2, "tol": 1e-8},
        "tol": 1e-14,
    }
    with open(os.path.join(HERE, "ctrap.json"), "w") as f:
        json.dump(doc, f, indent=1)


def lobpcg_diag():
    doc = {
        "source": "src/features/linalg/iterative.zig:80-203",
        "cases": [
            {"diag": [1.0, 2.0, 3.0], "nbands": 2, "max_iter": 20, "tol": 1e-8, "expected": [1.0, 2.0], "atol": 1e-6},
            {"diag": [1.0, 3.0, 5.0, 7.0], "nbands": 2, "max_iter": 20, "tol": 1e-8, "expected": [1.0, 3.0], "atol": 1e-6},
        ],
    }
    with open(os.path.join(HERE, "lobpcg_diag.json"), "w") as f:
        json.dump(doc, f, indent=1)


def lcg():
    s = 0x6F3D3CBE
    vals = []
    for _ in range(8):
        s = (s * 6364136223846793005 + 1) & ((1 << 64) - 1)
        vals.append((s >> 11) / 9007199254740992.0)
    doc = {"source": "src/features/linalg/lobpcg/common.zig:314-319; seed serial.zig:111", "seed": 0x6F3D3CBE, "first8": vals}
    with open(os.path.join(HERE, "lcg.json"), "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    local_potential_kats()
    fft_roundtrips()
    bessel()
    ctrap()
    lobpcg_diag()
    lcg()
    print("golden fixtures written to", HERE)
