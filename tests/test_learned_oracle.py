"""CPU checks of the learned preconditioner's float64 reference: analytic
gradients against central finite differences, and SPD-ness of M."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from oracle import learned_ref as lr  # noqa: E402
from cases import build_case  # noqa: E402


@pytest.fixture(scope="module")
def small(port_built):
    raw, nl, x, y, ax, ay, alpha, _ = build_case("tiny_macros")
    port = oracle.PortNetlist(nl)
    fx, fy = nl.floors()
    return nl, port.b2b_axis(True, x, fx, alpha, ax)


def test_gradients_match_finite_differences(small):
    nl, s = small
    params = lr.init_params(3)
    params["P"] *= 20.0  # away from tanh's linear regime
    graph = lr.Graph(nl)
    L, grads, _ = lr.loss_and_grad(params, s, nl, k=3, seed=5, graph=graph)
    rng = np.random.default_rng(0)
    for name in ("P", "Wb2", "Wc1", "Wa0", "ba1", "W_in", "b_in"):
        w = params[name]
        for _ in range(4):
            idx = tuple(int(rng.integers(0, k)) for k in w.shape)
            old = w[idx]
            eps = 1e-6 * max(1.0, abs(old))
            w[idx] = old + eps
            lp, _, _ = lr.loss_and_grad(params, s, nl, k=3, seed=5, graph=graph)
            w[idx] = old - eps
            lm, _, _ = lr.loss_and_grad(params, s, nl, k=3, seed=5, graph=graph)
            w[idx] = old
            fd = (lp - lm) / (2 * eps)
            g = grads[name][idx]
            assert abs(fd - g) <= 1e-5 * max(abs(fd), 1e-4), (name, idx, fd, g)


def test_preconditioner_is_spd(small):
    nl, s = small
    params = lr.init_params(1)
    params["P"] *= 50.0
    _, _, sv = lr.loss_and_grad(params, s, nl, k=1, seed=0)
    n = s["diag"].shape[0]
    M = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        M[:, j] = lr.apply_m(s, sv, e)
    assert np.allclose(M, M.T, atol=1e-12)
    assert np.linalg.eigvalsh(0.5 * (M + M.T)).min() > 0.0


def test_coarse_gradients_match_finite_differences(small):
    """The learned coarse vector's projection loss: analytic gradients of
    the head and of the trunk (on the topology features) against central
    differences."""
    nl, s = small
    params = lr.init_params(3)
    params["P"] *= 20.0
    params["wz"] *= 10.0  # a head whose output varies across cells
    graph = lr.Graph(nl)
    E = np.random.default_rng(1).standard_normal((2, nl.num_movable))
    L, grads, z = lr.coarse_loss_and_grad(params, s, nl, E, graph=graph)
    assert 0.0 <= L <= 1.0 and np.all(z > 0)
    rng = np.random.default_rng(2)
    checked = 0
    for name in ("bz", "wz", "Wh", "bh", "P", "Wb2", "Wa0", "W_in"):
        w = params[name]
        for _ in range(4):
            idx = tuple(int(rng.integers(0, k)) for k in w.shape)
            old = w[idx]
            eps = 1e-6 * max(1.0, abs(old))
            w[idx] = old + eps
            lp = lr.coarse_loss_and_grad(params, s, nl, E, graph=graph)[0]
            w[idx] = old - eps
            lm = lr.coarse_loss_and_grad(params, s, nl, E, graph=graph)[0]
            w[idx] = old
            fd = (lp - lm) / (2 * eps)
            g = grads[name][idx]
            assert abs(fd - g) <= 1e-4 * abs(fd) + 1e-10, (name, idx, fd, g)
            checked += abs(g) > 0
    assert checked >= 10


def test_untrained_coarse_head_is_constant(small):
    """The initial head (zero output weights' contribution aside) gives a
    coarse vector of ones: bias softplus^-1(1), output weights scaled down."""
    nl, s = small
    params = lr.init_params(4)
    params["wz"][:] = 0.0
    p, _ = lr.forward(params, lr.topo_features(nl), lr.Graph(nl))
    z, _ = lr.coarse_head(params, p, s)
    assert np.allclose(z, 1.0, rtol=0, atol=1e-12)
