"""Host side of the learned colouring: the numpy restatement of the policy that
the kernel evaluates agrees with the PyTorch network it is trained as, the flat
weight layout round-trips, and the clamp bounds the blue probability."""
from __future__ import annotations

import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def pol():
    return importlib.import_module("multicore-matching_b200.policy")


def _net(torch, pol):
    torch.manual_seed(3)
    return pol.make_net(torch)


def test_weight_layout_round_trips(pol):
    torch = pytest.importorskip("torch")
    net = _net(torch, pol)
    flat = pol._get(net)
    assert flat.shape == (pol.N_FLOATS,) and flat.dtype == np.float32
    other = _net(torch, pol)
    for p in other.parameters():
        p.data.zero_()
    pol._set(other, flat)
    assert np.array_equal(pol._get(other), flat)


def test_numpy_policy_matches_torch(pol):
    torch = pytest.importorskip("torch")
    net = _net(torch, pol)
    flat = pol._get(net)
    rng = np.random.default_rng(1)
    X = rng.uniform(0, 4, size=(512, 6)).astype(np.float32)
    ref = torch.sigmoid(net(torch.tensor(X)).squeeze(1)).clamp(pol.P_MIN, pol.P_MAX).detach().numpy()
    assert np.allclose(pol.policy_prob(flat, X), ref, atol=1e-5)


def test_clamp_bounds_probability(pol):
    w = np.zeros(pol.N_FLOATS, np.float32)
    X = np.ones((4, 6), np.float32)
    w[-1] = 40.0
    assert np.allclose(pol.policy_prob(w, X), 15 / 16)
    w[-1] = -40.0
    assert np.allclose(pol.policy_prob(w, X), 1 / 16)
    w[-1] = 0.0
    assert np.allclose(pol.policy_prob(w, X), 0.5)


def test_constant_policy_reproduces_the_barrier(pol):
    # the plain barrier's probability, as the constant policy's output
    w = pol.constant_policy(pol.P0)
    X = np.random.default_rng(0).uniform(0, 3, size=(16, 6)).astype(np.float32)
    assert np.allclose(pol.policy_prob(w, X), pol.P0, atol=1e-6)


def test_layout_matches_the_library(pol, mm):
    assert pol.N_FLOATS == mm.POLICY_FLOATS == 129


def test_fit_ips_stays_in_trust_region(pol):
    pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    X = rng.uniform(0, 4, size=(4096, 6)).astype(np.float32)
    c = (rng.random(4096) < pol.P0).astype(np.float32)
    # leaving is strongly favoured by blue where feature 0 is large: an
    # unconstrained fit would push those vertices to the clamp
    y = ((X[:, 0] > 2) & (c > 0.5)).astype(np.float32)
    w = pol.fit_ips(X, c, y, np.full(4096, pol.P0), delta=0.2, steps=300, device="cpu")
    p = pol.policy_prob(w, X)
    assert p[X[:, 0] > 3].mean() > pol.P0 + 0.1
    assert np.all(np.abs(p - pol.P0) < 0.2 + 0.03)


def test_es_refine_improves_a_quadratic(pol):
    target = np.linspace(-1, 1, pol.N_FLOATS).astype(np.float32)
    centre, best = pol.es_refine(lambda x: -float(((x - target) ** 2).sum()), np.zeros(pol.N_FLOATS, np.float32),
                                 iters=30, pairs=8, sigma=0.05, lr=0.05)
    start = float((target ** 2).sum())
    assert float(((centre - target) ** 2).sum()) < 0.5 * start
    assert float(((best - target) ** 2).sum()) < start


def test_hand_built_policy(pol):
    w = pol.hand_built(0, 2.0, 3.0)
    X = np.zeros((3, 6), np.float32)
    X[:, 0] = [3.0, 4.0, 2.0]
    p = pol.policy_prob(w, X)
    logit = np.log(pol.P0 / (1 - pol.P0))
    want = 1 / (1 + np.exp(-(logit + 2.0 * (X[:, 0] - 3.0))))
    assert np.allclose(p, np.clip(want, pol.P_MIN, pol.P_MAX), atol=1e-6)
