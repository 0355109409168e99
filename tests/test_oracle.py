"""CPU tests of the checker itself: the oracle restatement is pinned against the
reference's own code (live, where it is built) and against the committed
golden fixtures made from it."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from graphs_small import random_graph

BARRIER = 0x88B81733
K = [0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
     0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174]


def py_hash(v: int, r: int) -> int:
    """Independent Python statement of the colouring hash (src/matchgpu.cu:196-217)."""
    m = 0xFFFFFFFF
    h = [0x67452301, 0xefcdab89, 0x98badcfe, 0x10325476]
    a, b, c, d = h
    g = v
    for k in range(16):
        f = (b & c) | (~b & d)
        x = (a + f + K[k] + g) & m
        s = (7, 12, 17, 22)[k % 4]
        rot = ((x << s) | (x >> (32 - s))) & m
        a, b, c, d = d, (b + rot) & m, b, c
        h = [(h[0] + a) & m, (h[1] + b) & m, (h[2] + c) & m, (h[3] + d) & m]
        g = (g * r) & m
    return sum(h) & m


def test_hash_matches_independent_statement(orc):
    rng = np.random.default_rng(1)
    for _ in range(300):
        v, r = int(rng.integers(0, 2**31)), int(rng.integers(0, 2**31))
        assert orc.colour_hash(v, r) == py_hash(v, r)
    assert orc.colour_hash(0, 0) == py_hash(0, 0)


def test_rand_stream_is_glibc(mm, orc):
    for seed in (1, 7, 12345):
        assert np.array_equal(orc.rand_seeds(seed, 64), mm.rand_seeds(seed, 64))


def test_oracle_reproduces_golden(mm, orc, golden):
    graphs = {}
    checked = 0
    for c in golden.cases():
        if c["graph"] not in graphs:
            graphs[c["graph"]] = golden.graph(mm, c["graph"])
        g = graphs[c["graph"]]
        seeds = orc.rand_seeds(c["seed"], 256)
        m, rounds, _ = orc.match(g, c["type"], seeds, c["barrier"])
        assert rounds == c["rounds"], c["key"]
        want = golden.match(c["key"])
        if want is not None:
            assert np.array_equal(m, want), c["key"]
        assert hashlib.sha256(m.astype(np.int32).tobytes()).hexdigest() == c["sha256"], c["key"]
        if c["type"] in (7, 9):
            # the reference's next rand() value is the first one the matcher did not draw
            assert seeds[rounds] == c["next_rand"], c["key"]
        checked += 1
    assert checked > 300


def test_oracle_is_thread_count_invariant(mm, orc):
    g = mm.Graph.rmat(12, 16, seed=5)
    seeds = orc.rand_seeds(3)
    for t in (7, 9):
        a = orc.match(g, t, seeds, BARRIER, nthreads=1)
        b = orc.match(g, t, seeds, BARRIER, nthreads=8)
        assert a[1] == b[1] and np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])


def test_oracle_results_are_valid_and_maximal(mm, orc):
    for g in (mm.Graph.grid(64, 48), mm.Graph.rgg(3000, 13.0, seed=2), mm.Graph.er(3000, 8.0, seed=4)):
        seeds = orc.rand_seeds(11)
        for t in (7, 9):
            m, _, _ = orc.match(g, t, seeds, BARRIER)
            chk = orc.check(g, m)
            assert chk["valid"] and chk["matchable"] == 0
            assert set(np.unique(m[m < 4]).tolist()) <= {2}


def test_checker_flags_planted_mistakes(mm, orc):
    g = mm.Graph.grid(16, 16)
    m, _, _ = orc.match(g, 7, orc.rand_seeds(1), BARRIER)
    matched = np.nonzero(m >= 4)[0]
    bad = m.copy()
    bad[matched[0]] = 2  # partner left alone
    assert not orc.check(g, bad)["valid"]
    bad = m.copy()
    v = int(matched[0])
    far = int(np.nonzero(m >= 4)[0][-1])
    bad[far] = m[v]  # third holder of one match value
    assert not orc.check(g, bad)["valid"]
    bad = m.copy()
    bad[bad >= 4] = 2  # valid but not maximal
    chk = orc.check(g, bad)
    assert chk["valid"] and chk["matchable"] > 0


@pytest.mark.skipif("not __import__('oracle').ref_available()")
def test_checker_counts_equal_reference(mm, orc):
    """Pin of the restated testMatching counters against the reference's own,
    on matchings broken in each of its ways (the walk over values sorted by
    match value shifts after an unpaired vertex; the counters must follow it).
    Where a value has three or more holders the reference's order among them
    is std::sort's, so 'invalid' is compared only when no value has."""
    rng = np.random.default_rng(4)
    for g in (mm.Graph.grid(16, 16), mm.Graph.rmat(10, 8, seed=2), mm.Graph.er(300, 5.0, seed=3)):
        m, _, _ = orc.match(g, 9, orc.rand_seeds(7), BARRIER)
        cases = [m]
        for trial in range(12):
            x = m.copy()
            idx = rng.choice(g.n, size=1 + trial % 5, replace=False)
            x[idx] = rng.integers(-2, g.n + 8, size=len(idx))
            cases.append(x)
        for x in cases:
            got, want = orc.check(g, x), orc.ref_check_counts(g, x)
            vals, counts = np.unique(x[x >= 4], return_counts=True)
            keys = ("valid", "under", "multi", "matchable") + (("invalid",) if (counts < 3).all() else ())
            for k in keys:
                assert got[k] == want[k], (g.name, k, got, want)


@pytest.mark.skipif("not __import__('oracle').ref_available()")
def test_oracle_equals_reference_live(mm, orc):
    """Live pin: restatement vs the reference's TBB matchers on fresh graphs."""
    rng = np.random.default_rng(77)
    cases = [mm.Graph.rgg(20000, 13.0, seed=9), mm.Graph.rmat(13, 16, seed=2), mm.Graph.grid(100, 37)]
    for i in range(40):
        cases.append(random_graph(rng, int(rng.integers(1, 60)), avg_deg=float(rng.uniform(0.5, 6)),
                                  symmetric=bool(i % 2), gaps=bool(i % 3 == 0), shuffle_ranges=bool(i % 4 == 0),
                                  empty_reversed=0.2 if i % 5 == 0 else 0.0, dup=0.1, loops=0.1))
    for g in cases:
        for seed in (5, 999):
            seeds = orc.rand_seeds(seed, 256)
            for gpu_t, ref_t, fixed in ((6, 10, True), (7, 10, False), (8, 11, True), (9, 11, False)):
                want, _, nxt = orc.ref_run(g, ref_t, BARRIER, seed, fixed_rounds=fixed)
                got, rounds, _ = orc.match(g, gpu_t, seeds, BARRIER)
                assert np.array_equal(got, want)
                if not fixed:
                    assert seeds[rounds] == nxt
