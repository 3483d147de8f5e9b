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
