"""Learned colouring (mm_match_policy): whatever the policy, the result must be
a valid matching, maximal for the maximal types (checked with the oracle's
restatement of testMatching); the trace must hold one well-formed row per
coloured vertex and round.  The policy is not the reference's path (mm_match
is), so there is no bit-exact comparison here."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _policies(mm):
    rng = np.random.default_rng(0)
    yield np.zeros(mm.POLICY_FLOATS, np.float32)  # p = 1/2 everywhere
    w = np.zeros(mm.POLICY_FLOATS, np.float32)
    w[-1] = 2.5  # mostly blue (p = 0.92): slow but within the round cap
    yield w
    yield (rng.standard_normal(mm.POLICY_FLOATS) * 0.5).astype(np.float32)


@pytest.mark.parametrize("type_", [6, 7, 8, 9])
def test_policy_matchings_are_valid_and_maximal(mm, orc, torch_cuda, type_):
    seeds = orc.rand_seeds(12345, 256)
    for g in (mm.Graph.rgg(1 << 12, 13.0, seed=4), mm.Graph.rmat(12, 16, seed=2), mm.Graph.grid(40, 30)):
        with mm.DeviceGraph(g, device=0) as dg:
            for mlp in _policies(mm):
                out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
                rounds = dg.match_policy(type_, seeds, out.data_ptr(), mlp, 1.0)
                m = out.cpu().numpy()
                chk = orc.check(g, m)
                assert chk["valid"], (g.name, type_, chk)
                if type_ in (7, 9):
                    assert chk["matchable"] == 0 and rounds <= 255, (g.name, chk)
                else:
                    assert rounds == 20


def test_policy_trace_rows(mm, orc, torch_cuda):
    g = mm.Graph.rgg(1 << 12, 13.0, seed=9)
    seeds = orc.rand_seeds(5, 256)
    w = np.zeros(mm.POLICY_FLOATS, np.float32)
    with mm.DeviceGraph(g, device=0) as dg:
        rounds_cap = 40
        tr = torch_cuda.full((rounds_cap * g.n * 8,), float("nan"), dtype=torch_cuda.float32, device="cuda")
        out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        rounds = dg.match_policy(9, seeds, out.data_ptr(), w, 2.0, tr.data_ptr(), rounds_cap)
        t = tr.view(rounds_cap, g.n, 8).cpu().numpy()
        m = out.cpu().numpy()
    coloured = ~np.isnan(t[:, :, 6])
    assert coloured[0].all()  # every vertex is coloured in round 0
    rows = t[coloured]
    assert set(np.unique(rows[:, 6])) <= {0.0, 1.0} and set(np.unique(rows[:, 7])) <= {0.0, 1.0}
    assert np.allclose(rows[:, 5], 2.0 / 16)  # the level feature
    for r in range(rounds_cap):  # the round feature saturates at 32 rounds
        assert np.allclose(t[r][coloured[r]][:, 4], min(r, 32) / 32)
    deg = g.degrees()
    assert np.allclose(t[0, :, 0], np.log2(1 + deg), atol=1e-5)
    assert np.all(t[0, :, 1] == 0.0)  # no previous round
    assert set(np.unique(rows[:, 1])) <= {0.0, 0.5, 1.0}  # previous role
    # a vertex red in round r has role 0 in round r + 1
    for r in range(rounds_cap - 1):
        both = coloured[r] & coloured[r + 1]
        assert np.all(t[r + 1, :, 1][both & (t[r, :, 6] == 0.0)] == 0.0)
        assert np.all(t[r + 1, :, 1][both & (t[r, :, 6] == 1.0)] > 0.0)
    # every vertex that left the active set (matched, or retired with match
    # value 2) is marked in exactly one round, survivors in none
    marks = np.nansum(t[:, :, 7], axis=0)
    assert np.array_equal(marks, ((m >= 4) | (m == 2)).astype(np.float64))
    # a vertex is marked in a round in which it was coloured
    assert not np.isnan(t[:, :, 6][t[:, :, 7] == 1]).any()
    assert rounds <= rounds_cap


@pytest.mark.parametrize("type_", [6, 7, 8, 9])
def test_zero_policy_gives_the_plain_matching(mm, orc, torch_cuda, type_):
    """With all weights 0 the policy's probability is exactly 1/2, the select
    barrier 0x80000000: the colours are the plain method's, and retiring
    vertices whose neighbours are all matched early changes no matched pair, only the
    rounds (maximal types) and the match value of unmatched vertices (2 for
    retired ones, their colour for survivors of the fixed-round types)."""
    seeds = orc.rand_seeds(777, 256)
    w = np.zeros(mm.POLICY_FLOATS, np.float32)
    for g in (mm.Graph.rgg(1 << 13, 13.0, seed=5), mm.Graph.rmat(13, 16, seed=6), mm.Graph.grid(50, 40)):
        with mm.DeviceGraph(g, device=0) as dg:
            a = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
            b = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
            r_plain = dg.match_device(type_, seeds, a.data_ptr(), 0x80000000)
            r_pol = dg.match_policy(type_, seeds, b.data_ptr(), w, 0.0, barrier=0x80000000)
            ma, mb = a.cpu().numpy(), b.cpu().numpy()
            assert np.array_equal(ma >= 4, mb >= 4), g.name
            assert np.array_equal(ma[ma >= 4], mb[mb >= 4]), g.name
            if type_ in (7, 9):
                assert np.array_equal(ma, mb) and r_pol <= r_plain, (g.name, r_pol, r_plain)


@pytest.mark.parametrize("type_", [6, 7, 8, 9])
def test_zero_policy_is_the_plain_matching_off_the_symmetric_path(mm, orc, torch_cuda, type_):
    """On a CSR that does not take the symmetric path (asymmetric entries,
    duplicates, self-loops, shuffled and gapped ranges) nothing retires early,
    so the zero policy (p = 1/2 exactly, barrier 0x80000000) gives exactly the
    plain result: every match value and the round count."""
    from graphs_small import random_graph

    seeds = orc.rand_seeds(4242, 256)
    w = np.zeros(mm.POLICY_FLOATS, np.float32)
    rng = np.random.default_rng(17)
    for i in range(6):
        g = random_graph(rng, int(rng.integers(50, 3000)), avg_deg=float(rng.uniform(1.0, 8.0)),
                         symmetric=False, shuffle_ranges=i % 2 == 0, gaps=i % 3 == 0)
        with mm.DeviceGraph(g, device=0) as dg:
            a = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
            b = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
            r_plain = dg.match_device(type_, seeds, a.data_ptr(), 0x80000000)
            r_pol = dg.match_policy(type_, seeds, b.data_ptr(), w, 0.0, barrier=0x80000000)
            ma, mb = a.cpu().numpy(), b.cpu().numpy()
        assert r_pol == r_plain and np.array_equal(ma, mb), (i, g.n)
        assert orc.check(g, mb)["valid"]


def test_policy_on_a_batch_matches_every_graph(mm, orc, torch_cuda):
    """On a batch every graph's slice is a valid maximal matching of that graph,
    in its own numbering."""
    seeds = orc.rand_seeds(99, 256)
    graphs = [mm.Graph.rgg(2000, 13.0, seed=1), mm.Graph.grid(30, 20), mm.Graph.rmat(11, 16, seed=4),
              mm.Graph.rgg(500, 6.0, seed=2)]
    u, off = mm.Graph.union(graphs)
    rng = np.random.default_rng(5)
    mlp = (rng.standard_normal(mm.POLICY_FLOATS) * 0.5).astype(np.float32)
    with mm.DeviceGraph(u, device=0) as dg:
        dg.set_batch(off)
        out = torch_cuda.empty(u.n, dtype=torch_cuda.int32, device="cuda")
        rounds = dg.match_policy(9, seeds, out.data_ptr(), mlp, 1.0)
        m = out.cpu().numpy()
    assert rounds <= 255
    for i, g in enumerate(graphs):
        chk = orc.check(g, m[off[i]:off[i + 1]])
        assert chk["valid"] and chk["matchable"] == 0, (i, g.name, chk)


def test_policy_that_ignores_its_features_is_constant(mm, orc, torch_cuda):
    """Random hidden weights behind an all-zero output layer give the same
    probability everywhere, so the same matching as the all-zero policy."""
    seeds = orc.rand_seeds(31, 256)
    rng = np.random.default_rng(8)
    w = (rng.standard_normal(mm.POLICY_FLOATS) * 2.0).astype(np.float32)
    w[6 * 16 + 16:] = 0.0  # W2 and b2
    g = mm.Graph.rgg(1 << 13, 13.0, seed=12)
    with mm.DeviceGraph(g, device=0) as dg:
        a = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        b = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        ra = dg.match_policy(9, seeds, a.data_ptr(), w, 0.0)
        rb = dg.match_policy(9, seeds, b.data_ptr(), np.zeros(mm.POLICY_FLOATS, np.float32), 0.0)
        assert ra == rb and np.array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_policy_mlp_device_matches_host(mm, orc, torch_cuda):
    """The MLP the colouring evaluates on the device gives, from the traced
    features, the same colour as a numpy evaluation of the same weights
    (policy.policy_prob): blue iff hash < p * 2^32, except where the hash lies
    within a band of the threshold that fp32 rounding can cross."""
    import importlib

    pol = importlib.import_module("multicore_matching_b200.policy")
    rng = np.random.default_rng(11)
    mlp = (rng.standard_normal(mm.POLICY_FLOATS) * 0.6).astype(np.float32)
    g = mm.Graph.rgg(1 << 12, 13.0, seed=3)
    seeds = orc.rand_seeds(77, 256)
    cap = 48
    with mm.DeviceGraph(g, device=0) as dg:
        tr = torch_cuda.full((cap * g.n * 8,), float("nan"), dtype=torch_cuda.float32, device="cuda")
        out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        rounds = dg.match_policy(9, seeds, out.data_ptr(), mlp, 1.0, tr.data_ptr(), cap)
        t = tr.view(cap, g.n, 8).cpu().numpy()[: min(rounds, cap)]
    rr, vv = np.nonzero(~np.isnan(t[:, :, 6]))
    rows = t[rr, vv]
    p = pol.policy_prob(mlp.astype(np.float64), rows[:, :6].astype(np.float64))
    thr = p * 4294967296.0
    h = np.array([orc.colour_hash(int(v), int(seeds[r])) for r, v in zip(rr, vv)], dtype=np.float64)
    band = np.abs(h - thr) <= 4294967296.0 * 1e-5
    want = (h < thr).astype(np.float32)
    assert len(rows) > 5000 and band.mean() < 0.01
    assert np.array_equal(rows[~band, 6], want[~band]), int((rows[~band, 6] != want[~band]).sum())


@pytest.mark.parametrize("type_", [6, 7, 8, 9])
def test_constant_policy_finish_phase_equals_its_rounds(mm, orc, torch_cuda, type_):
    """A policy that ignores its features hands the late rounds to the finish
    kernel, which plays them under the policy's threshold and the retirement
    rule of the round kernel (a red vertex of at most 128 entries whose
    neighbours are all matched leaves from round 3 on).  Every match value and
    the round count must equal those of the round kernel playing every round
    itself (finish phase off), on the symmetric graphs that take that path and
    on a batch."""
    import importlib

    pol = importlib.import_module("multicore_matching_b200.policy")
    seeds = orc.rand_seeds(2024, 256)
    policies = [np.zeros(mm.POLICY_FLOATS, np.float32), pol.load_policy(), pol.constant_policy(0.7)]
    graphs = [mm.Graph.rgg(1 << 13, 13.0, seed=21), mm.Graph.rmat(13, 16, seed=22), mm.Graph.grid(64, 48),
              mm.Graph.er(1 << 12, 8.0, seed=23)]
    u, off = mm.Graph.union(graphs[:3])
    for g, batch in [(x, None) for x in graphs] + [(u, off)]:
        with mm.DeviceGraph(g, device=0) as dg:
            if batch is not None:
                dg.set_batch(batch)
            for w in policies:
                a = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
                b = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
                dg.tune(finish_div=0)
                ra = dg.match_policy(type_, seeds, a.data_ptr(), w, 1.0)
                dg.tune(finish_div=-1)
                rb = dg.match_policy(type_, seeds, b.data_ptr(), w, 1.0)
                ma, mb = a.cpu().numpy(), b.cpu().numpy()
                assert ra == rb and np.array_equal(ma, mb), (g.name, type_, ra, rb, int((ma != mb).sum()))
                if batch is None:
                    chk = orc.check(g, ma)
                    assert chk["valid"] and (type_ in (6, 8) or chk["matchable"] == 0), (g.name, chk)
