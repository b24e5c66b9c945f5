"""CPU: the host side of the learned-preconditioner pipeline (dft-zig_b200/learn.py) against the
oracle network (oracle/learned.py): the untrained and alpha = 0 networks are Teter-Payne-Allan,
the iteration input can be removed, and the host loss of a fixed preconditioner equals the
oracle's loss for the same multiplier."""
import importlib

import numpy as np
import pytest

from oracle import learned


@pytest.fixture(scope="module")
def learn():
    import dftzig_loader

    dftzig_loader.load()
    return importlib.import_module("dftzig_b200.learn")


def _u(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(-3.0, 4.0, n), rng.uniform(-13.0, 5.0, n), rng.uniform(0.0, 2.0, n)], axis=1)


def test_untrained_network_is_tpa(learn):
    p = learn.init_params(seed=3)
    u = _u(500, 1)
    x = np.maximum(np.exp(u[:, 0]) - 0.05, 0.0)
    assert np.allclose(learned.multiplier(p, u), learned.tpa(x), rtol=0, atol=1e-15)


def test_scale_output_interpolates_between_tpa_and_the_network(learn):
    p = learned.init_params(seed=2).astype(np.float32)
    p[-65:] = np.random.default_rng(4).normal(0.0, 0.3, 65)  # a nonzero output layer
    u = _u(400, 2)
    z = learned.forward(p, u)[0]
    assert np.array_equal(learn.scale_output(p, 1.0), p)
    assert np.abs(learned.forward(learn.scale_output(p, 0.0), u)[0]).max() == 0.0
    assert np.allclose(learned.forward(learn.scale_output(p, 0.5), u)[0], 0.5 * z, rtol=1e-6, atol=1e-6)


def test_without_iteration_input_makes_the_network_ignore_t(learn):
    p = learned.init_params(seed=5).astype(np.float32)
    p[-65:] = np.random.default_rng(6).normal(0.0, 0.3, 65)
    off, feat, cc, w, dnorm = learned.random_problem(seed=1)
    s, q = learn.without_iteration_input({"off": off, "feat": feat.astype(np.float32), "cc": cc, "w": w, "dnorm": dnorm}, p)
    assert np.all(s["feat"][:, 2] == 0.0)
    u = _u(300, 3)
    u2 = u.copy()
    u2[:, 2] = 1.7
    assert np.array_equal(learned.forward(q, u)[0], learned.forward(q, u2)[0])


def test_fixed_tpa_loss_matches_the_oracle_loss(learn):
    off, feat, cc, w, dnorm = learned.random_problem(seed=8)
    n = int(off[-1])
    samples = {"off": off, "feat": feat.astype(np.float32), "cc": cc, "w": w, "dnorm": dnorm,
               "kin": np.zeros(n), "lam": np.zeros(len(off) - 1)}  # the TPA form reads only feat
    L_host = learn.fixed_loss(samples, "tpa")
    L_oracle, _ = learned.loss_grad(learn.init_params(seed=0), off, feat.astype(np.float32).astype(np.float64), cc, w, dnorm)
    assert abs(L_host - L_oracle) < 1e-12
