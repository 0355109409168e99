"""Host-side graph helpers of the package, on the CPU: the disjoint union that
mm_graph_set_batch takes (vertex and entry ids shifted, per-graph offsets),
and pair-hash weights (both entries of an edge weigh the same)."""
from __future__ import annotations

import numpy as np
import pytest


def test_union_slices_are_the_graphs(mm):
    a = mm.Graph.grid(5, 4)
    b = mm.Graph.rgg(300, 6.0, seed=3)
    empty = mm.Graph(0, np.zeros((0, 2), np.int32), np.zeros(0, np.int32), None, "empty")
    unit = mm.Graph(3, np.array([[0, 1], [1, 3], [3, 4]], np.int32), np.array([1, 0, 2, 1], np.int32), None, "unit")
    u, off = mm.Graph.union([a, empty, b, unit])
    assert list(off) == [0, a.n, a.n, a.n + b.n, a.n + b.n + 3]
    assert u.n == a.n + b.n + 3 and u.nnz == a.nnz + b.nnz + 4
    e0 = 0
    for g, v0 in zip((a, empty, b, unit), off[:-1]):
        r = u.ranges[v0:v0 + g.n].astype(np.int64) - e0
        assert np.array_equal(r, g.ranges)
        assert np.array_equal(u.nbrs[e0:e0 + g.nnz] - v0, g.nbrs)
        want_w = np.ones(g.nnz, np.float32) if g.weights is None else g.weights
        assert np.array_equal(u.weights[e0:e0 + g.nnz], want_w)
        # no entry leaves its graph
        assert ((u.nbrs[e0:e0 + g.nnz] >= v0) & (u.nbrs[e0:e0 + g.nnz] < v0 + g.n)).all()
        e0 += g.nnz


def test_union_rejects_int32_overflow(mm):
    class Big:  # sizes only: the check comes before any array is built
        n = 1 << 30
        nnz = 0
    with pytest.raises(ValueError):
        mm.Graph.union([Big(), Big()])


def test_pair_weights_are_symmetric(mm):
    g = mm.Graph.er(2000, 6.0, seed=5).with_pair_weights(seed=2)
    deg = g.degrees()
    owner = np.repeat(np.arange(g.n), deg)
    assert (g.weights > 0).all() and (g.weights <= 1).all()
    fwd = owner.astype(np.int64) * g.n + g.nbrs
    rev = g.nbrs.astype(np.int64) * g.n + owner
    of, orv = np.argsort(fwd), np.argsort(rev)
    assert np.array_equal(fwd[of], rev[orv])
    assert np.array_equal(g.weights[of], g.weights[orv])
    # another seed, other weights; the same seed, the same weights
    assert not np.array_equal(g.weights, g.with_pair_weights(seed=3).weights)
    assert np.array_equal(g.weights, g.with_pair_weights(seed=2).weights)
