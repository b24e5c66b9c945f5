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
