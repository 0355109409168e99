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
