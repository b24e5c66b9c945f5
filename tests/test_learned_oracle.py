"""CPU: the learned-preconditioner oracle (oracle/learned.py) against finite differences, and the
TPA limit values."""
import numpy as np

from oracle import learned


def test_tpa_limits():
    assert learned.tpa(np.array([0.0]))[0] == 1.0
    x = np.array([100.0, 1000.0])
    # K(x) -> 8x^3 / 16x^4 = 1 / (2x) for large x
    assert np.allclose(learned.tpa(x) * 2 * x, 1.0, rtol=0.02)


def test_loss_gradient_matches_finite_differences():
    off, feat, cc, w, dnorm = learned.random_problem(seed=3)
    p = learned.init_params(seed=1)
    L, g = learned.loss_grad(p, off, feat, cc, w, dnorm)
    assert 0.0 <= L <= 1.0
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(learned.NPARAM, 40, replace=False), [learned.NPARAM - 1]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (learned.loss_grad(p + e, off, feat, cc, w, dnorm)[0] - learned.loss_grad(p - e, off, feat, cc, w, dnorm)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_loss_is_scale_free():
    off, feat, cc, w, dnorm = learned.random_problem(seed=4)
    p = learned.init_params(seed=2)
    L1, _ = learned.loss_grad(p, off, feat, cc, w, dnorm)
    L2, _ = learned.loss_grad(p, off, feat, 7.0 * cc, 49.0 * w, dnorm)
    assert abs(L1 - L2) < 1e-12


def test_table_inference_error_bound_for_shipped_weights():
    """The solver evaluates the network through a table over (u0, u1) with bilinear interpolation
    (csrc/learned.cu: k_mlp_table, k_precondition_lut).  With the grid the CUDA source declares, the
    interpolated z of the shipped weights stays within 1e-4 of the network (documented: 5e-5) at
    random points of the range real inputs take, for several iteration inputs t."""
    import os
    import re

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "dft-zig_b200", "csrc", "learned.cu")).read()
    n0, n1 = (int(v) for v in re.search(r"kLutN0 = (\d+), kLutN1 = (\d+);", src).groups())
    lo0, hi0, lo1, hi1 = (float(v) for v in re.search(
        r"kLutU0 = ([-\d.]+)f, kLutU0Hi = ([-\d.]+)f, kLutU1 = ([-\d.]+)f, kLutU1Hi = ([-\d.]+)f;", src).groups())
    with np.load(os.path.join(root, "dft-zig_b200", "weights", "precond_mlp.npz")) as z:
        p = np.asarray(z["params"], dtype=np.float64)
    g0, g1 = np.linspace(lo0, hi0, n0), np.linspace(lo1, hi1, n1)
    rng = np.random.default_rng(7)
    u0 = rng.uniform(np.log(0.05), 4.5, 50000)
    u1 = rng.uniform(np.log(1e-6), 5.5, 50000)
    for t in (0.0, 7.0, 40.0):
        G0, G1 = np.meshgrid(g0, g1, indexing="ij")
        grid = np.stack([G0.ravel(), G1.ravel(), np.full(G0.size, min(t / 20.0, 2.0))], axis=1)
        table = learned.forward(p, grid)[0].reshape(n0, n1)
        f0, f1 = (u0 - lo0) * (n0 - 1) / (hi0 - lo0), (u1 - lo1) * (n1 - 1) / (hi1 - lo1)
        i0, i1 = np.floor(f0).astype(int), np.floor(f1).astype(int)
        a, c = f0 - i0, f1 - i1
        z0 = table[i0, i1] + c * (table[i0, i1 + 1] - table[i0, i1])
        z1 = table[i0 + 1, i1] + c * (table[i0 + 1, i1 + 1] - table[i0 + 1, i1])
        zi = z0 + a * (z1 - z0)
        u = np.stack([u0, u1, np.full_like(u0, min(t / 20.0, 2.0))], axis=1)
        assert np.abs(zi - learned.forward(p, u)[0]).max() < 1e-4
