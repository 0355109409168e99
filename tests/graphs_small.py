"""Small adversarial CSR graphs for CPU-side equivalence tests.

They exercise every input the reference's kernels accept: duplicate and
self-loop entries, one-directional entries, neighbour lists that are not
contiguous, not in vertex order or empty/reversed, and weights with ties,
signed zeros, values at and below -1, NaN and infinities.
"""
from __future__ import annotations

import numpy as np

SPECIAL_WEIGHTS = np.array([0.5, 0.5, 1.0, 0.0, -0.0, -1.0, -2.0, -0.5, np.nan, np.inf, -np.inf,
                            1e-45, 3.0, 3.0, 0.25], dtype=np.float32)


class SmallGraph:
    def __init__(self, n, ranges, nbrs, weights):
        self.n = n
        self.ranges = np.asarray(ranges, dtype=np.int32).reshape(n, 2)
        self.nbrs = np.asarray(nbrs, dtype=np.int32)
        self.weights = None if weights is None else np.asarray(weights, dtype=np.float32)

    @property
    def nnz(self):
        return int(self.nbrs.shape[0])


def random_graph(rng: np.random.Generator, n: int, avg_deg: float = 3.0, symmetric: bool = True,
                 dup: float = 0.05, loops: float = 0.03, gaps: bool = False, shuffle_ranges: bool = False,
                 empty_reversed: float = 0.0, special_weights: bool = True, sort_lists: bool = False) -> SmallGraph:
    m = int(n * avg_deg / 2)
    lists = [[] for _ in range(n)]
    for _ in range(m):
        u, v = int(rng.integers(n)), int(rng.integers(n))
        if u == v and rng.random() > loops:
            continue
        wt = (SPECIAL_WEIGHTS[rng.integers(len(SPECIAL_WEIGHTS))] if special_weights and rng.random() < 0.3
              else np.float32(rng.integers(1, 8) / 4))
        w2 = wt if (symmetric or rng.random() < 0.5) else np.float32(rng.integers(1, 8) / 4)
        lists[u].append((v, wt))
        if u != v and (symmetric or rng.random() < 0.6):
            lists[v].append((u, w2))
        if rng.random() < dup:
            lists[u].append((v, np.float32(rng.integers(1, 8) / 4)))
    for l in lists:
        rng.shuffle(l)
        if sort_lists:  # ascending neighbour ids, duplicates kept in their shuffled order
            l.sort(key=lambda e: e[0])
    order = np.arange(n)
    if shuffle_ranges:
        rng.shuffle(order)
    nbrs, wts = [], []
    ranges = np.zeros((n, 2), np.int64)
    for v in order:
        if gaps and rng.random() < 0.3:
            k = int(rng.integers(1, 3))
            nbrs += [int(rng.integers(n)) for _ in range(k)]
            wts += [np.float32(9.0)] * k
        b = len(nbrs)
        for (u, wt) in lists[v]:
            nbrs.append(u)
            wts.append(wt)
        ranges[v] = (b, len(nbrs))
        if empty_reversed and rng.random() < empty_reversed and b == len(nbrs):
            ranges[v] = (b + 1, b)  # reversed range: degree 0
    return SmallGraph(n, ranges, np.array(nbrs, np.int32), np.array(wts, np.float32))
