"""CPU design check: the push-path reformulation equals the oracle on
adversarial inputs (see tests/push_model.py)."""
from __future__ import annotations

import numpy as np

from graphs_small import random_graph
from push_model import push_match, reverse_keys, reverse_keys_sorted


def test_push_model_equals_oracle(orc):
    rng = np.random.default_rng(12)
    total = 0
    for it in range(120):
        n = int(rng.integers(1, 40))
        g = random_graph(rng, n, avg_deg=float(rng.uniform(0.5, 6)), symmetric=bool(rng.random() < 0.6),
                         gaps=bool(rng.random() < 0.3), shuffle_ranges=bool(rng.random() < 0.3),
                         empty_reversed=0.2 if rng.random() < 0.3 else 0.0, dup=0.1, loops=0.1)
        seeds = orc.rand_seeds(int(rng.integers(1, 1000)))
        for barrier in (0x88B81733, 0x40000000, 0, 0xFFFFFFFF):
            for t in (6, 7, 8, 9):
                want, rounds, _ = orc.match(g, t, seeds, barrier)
                got, got_rounds = push_match(g, t, seeds, barrier, orc.colour_hash)
                assert got_rounds == rounds
                assert np.array_equal(got, want), (it, t, hex(barrier))
                total += 1
    assert total == 120 * 16


def test_sorted_reverse_key_build_equals_pair_definition():
    """k_revkey_sorted's indexing (chunked owners, shared prefix table or bounded
    search, lower bound in the neighbour's list) gives the reverse keys of their
    definition on sorted lists, and reports every unsorted graph."""
    rng = np.random.default_rng(77)
    seen_unsorted = 0
    for it in range(150):
        n = int(rng.integers(1, 60))
        sort = rng.random() < 0.8
        g = random_graph(rng, n, avg_deg=float(rng.uniform(0.3, 7)), symmetric=bool(rng.random() < 0.6),
                         gaps=bool(rng.random() < 0.3), shuffle_ranges=bool(rng.random() < 0.3),
                         empty_reversed=0.3 if rng.random() < 0.3 else 0.0, dup=0.1, loops=0.1, sort_lists=sort)
        if rng.random() < 0.3:  # long runs of isolated vertices inside a chunk
            g.ranges[rng.random(n) < 0.5] = [0, 0]
        w = g.weights
        chunk = int(rng.choice([1, 2, 3, 8, 2048]))
        for weighted in (False, True):
            want = reverse_keys(n, g.ranges, g.nbrs, w, weighted)
            got = reverse_keys_sorted(n, g.ranges, g.nbrs, w, weighted, chunk)
            lists_sorted = all(np.all(np.diff(g.nbrs[b:e].astype(np.int64)) >= 0) for b, e in g.ranges if e > b)
            if lists_sorted:
                assert got == want, (it, chunk, weighted)
            else:
                assert got is None
                seen_unsorted += 1
    assert seen_unsorted > 0


def symmetric_graph(rng, n, avg_deg, loops=0.05, special=True):
    """A CSR that takes the symmetric path: contiguous, strictly increasing lists,
    every entry's transpose present with the same weight (self-loops once)."""
    from graphs_small import SPECIAL_WEIGHTS, SmallGraph

    pairs = {}
    for _ in range(int(n * avg_deg / 2)):
        u, v = int(rng.integers(n)), int(rng.integers(n))
        if u == v and rng.random() > loops:
            continue
        a, b = min(u, v), max(u, v)
        if (a, b) in pairs:
            continue
        pairs[(a, b)] = (SPECIAL_WEIGHTS[rng.integers(len(SPECIAL_WEIGHTS))] if special and rng.random() < 0.3
                         else np.float32(rng.integers(1, 8) / 4))
    lists = [[] for _ in range(n)]
    for (a, b), wt in pairs.items():
        lists[a].append((b, wt))
        if a != b:
            lists[b].append((a, wt))
    nbrs, wts, ranges = [], [], np.zeros((n, 2), np.int64)
    for v in range(n):
        ranges[v, 0] = len(nbrs)
        for u, wt in sorted(lists[v], key=lambda e: e[0]):
            nbrs.append(u)
            wts.append(wt)
        ranges[v, 1] = len(nbrs)
    return SmallGraph(n, ranges, np.array(nbrs, np.int32), np.array(wts, np.float32))


def test_finish_phase_model_equals_oracle(orc):
    """The finish phase (components played on their own from the round the
    active set is small enough) gives the oracle's matching and round count,
    whether it completes or is called off (small limits force both)."""
    import push_model

    outcomes = {"done": 0, "off": 0}
    model = push_model.finish_model

    def counted(*a, **k):
        r = model(*a, **k)
        outcomes["done" if r is not None else "off"] += 1
        return r

    push_model.finish_model = counted
    try:
        rng = np.random.default_rng(5)
        for it in range(60):
            n = int(rng.integers(2, 90))
            g = symmetric_graph(rng, n, float(rng.uniform(0.5, 5)))
            assert push_model.is_symmetric(g.n, g.ranges, g.nbrs, g.weights, True)
            seeds = orc.rand_seeds(int(rng.integers(1, 1000)))
            lim = [dict(div=1, members=32, entries=128, maxdeg=2048), dict(div=2, members=3, entries=4, maxdeg=4),
                   dict(div=12, members=32, entries=128, maxdeg=2048)][it % 3]
            for barrier in (0x88B81733, 0x40000000):
                for t in (6, 7, 8, 9):
                    want, rounds, _ = orc.match(g, t, seeds, barrier)
                    got, got_rounds = push_match(g, t, seeds, barrier, orc.colour_hash, finish=lim)
                    assert got_rounds == rounds, (it, t, hex(barrier))
                    assert np.array_equal(got, want), (it, t, hex(barrier))
    finally:
        push_model.finish_model = model
    assert outcomes["done"] > 100 and outcomes["off"] > 100, outcomes


def test_isolated_vertices_at_set_up_equal_oracle(orc):
    """Resolving the vertices without neighbours at set-up (the round kernel's
    rule on the symmetric path) gives the oracle's match values and round count:
    sparse symmetric graphs with many isolated vertices, barriers that keep
    vertices red for long (to the cap of the maximal loop), with and without the
    finish phase."""
    import push_model

    rng = np.random.default_rng(31)
    fin = dict(div=4, members=6, entries=16, maxdeg=12)
    checked = 0
    for it in range(40):
        n = int(rng.integers(1, 60))
        g = symmetric_graph(rng, n, float(rng.uniform(0.0, 1.5)))
        assert push_model.is_symmetric(g.n, g.ranges, g.nbrs, g.weights, True)
        seeds = orc.rand_seeds(int(rng.integers(1, 1000)))
        for barrier in (0x88B81733, 0x20000000, 0x02000000):
            for t in (6, 7, 8, 9):
                want, rounds, _ = orc.match(g, t, seeds, barrier)
                for f in (None, fin):
                    got, got_rounds = push_match(g, t, seeds, barrier, orc.colour_hash, finish=f, isolated=True)
                    assert got_rounds == rounds, (it, t, hex(barrier), f is None)
                    assert np.array_equal(got, want), (it, t, hex(barrier), f is None)
                    checked += 1
    assert checked == 40 * 3 * 4 * 2
