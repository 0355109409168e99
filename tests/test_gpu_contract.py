"""Contraction of a matched graph (mm_graph_contract) against a numpy restatement
of the same rules, and a multilevel chain down to 1% of the vertices.  The
contraction has no counterpart in the reference (it stops at the matching);
the rules checked here are the ones include/mm_match.h states."""
from __future__ import annotations

import numpy as np
import pytest

from graphs_small import random_graph

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def contract_ref(ranges, nbrs, w, match):
    """Coarse CSR: pairs merged into their smaller member's id order, entries mapped,
    self-loops dropped, parallel entries summed in double and rounded once."""
    n = len(match)
    ranges = np.asarray(ranges).reshape(-1, 2).astype(np.int64)
    match = np.asarray(match, dtype=np.int64)
    rep = np.where(match >= 4, match - 4, np.arange(n))
    first = rep == np.arange(n)
    cid = np.cumsum(first) - first
    cmap = cid[rep]
    nc = int(first.sum())
    deg = np.maximum(ranges[:, 1] - ranges[:, 0], 0)
    owner = np.repeat(np.arange(n), deg)
    pos = np.concatenate([np.arange(b, b + d) for (b, _), d in zip(ranges, deg)]) if n else np.zeros(0, np.int64)
    c = cmap[owner]
    cu = cmap[np.asarray(nbrs, dtype=np.int64)[pos]]
    ww = np.asarray(w, dtype=np.float64)[pos]
    keep = c != cu
    c, cu, ww = c[keep], cu[keep], ww[keep]
    order = np.lexsort((cu, c))
    c, cu, ww = c[order], cu[order], ww[order]
    if len(c):
        head = np.ones(len(c), bool)
        head[1:] = (c[1:] != c[:-1]) | (cu[1:] != cu[:-1])
        idx = np.nonzero(head)[0]
        sums = np.add.reduceat(ww, idx)
        c, cu = c[idx], cu[idx]
    else:
        sums = np.zeros(0)
    counts = np.bincount(c, minlength=nc)
    off = np.concatenate([[0], np.cumsum(counts)])
    return nc, np.stack([off[:-1], off[1:]], axis=1).astype(np.int32), cu.astype(np.int32), sums.astype(np.float32), cmap


def _check_contraction(mm, torch, dg, g, m):
    d = torch.from_numpy(np.ascontiguousarray(m, dtype=np.int32)).cuda()
    cmap = torch.empty(g.n, dtype=torch.int32, device="cuda")
    with dg.contract(d.data_ptr(), cmap.data_ptr()) as cg:
        r, nb, w = cg.to_host()
        nc, r_ref, nb_ref, w_ref, cmap_ref = contract_ref(np.asarray(g.ranges), g.nbrs, g.weights, m)
        assert cg.n == nc
        assert np.array_equal(r, r_ref)
        assert np.array_equal(nb, nb_ref)
        assert np.array_equal(w, w_ref)
        assert np.array_equal(cmap.cpu().numpy(), cmap_ref)


def test_contract_matches_restatement(mm, orc, torch_cuda):
    for g in (mm.Graph.grid(32, 32), mm.Graph.rgg(1 << 12, 13.0, seed=5), mm.Graph.rmat(12, 16, seed=4),
              mm.Graph.er(1 << 11, 8.0, seed=6)):
        seeds = orc.rand_seeds(12345, 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for t in (6, 9):
                m, _, _ = orc.match(g, t, seeds, BARRIER)
                _check_contraction(mm, torch_cuda, dg, g, m)


def test_contract_general_csr(mm, orc, torch_cuda):
    for seed in range(4):
        g = random_graph(np.random.default_rng(seed), 300, 5.0, symmetric=seed % 2 == 0, gaps=seed % 2 == 1,
                         shuffle_ranges=seed == 3, special_weights=False, sort_lists=seed == 0)
        with mm.DeviceGraph(g, device=0) as dg:
            m, _, _ = orc.match(g, 9, orc.rand_seeds(seed + 3, 256), BARRIER)
            _check_contraction(mm, torch_cuda, dg, g, m)


def test_contract_rejects_non_matching(mm, torch_cuda):
    g = mm.Graph.grid(8, 8)
    bad = np.zeros(g.n, dtype=np.int32)
    bad[5] = 4 + 9  # names vertex 9, which does not name it back
    d = torch_cuda.from_numpy(bad).cuda()
    with mm.DeviceGraph(g, device=0) as dg:
        with pytest.raises(mm.MatchError) as err:
            dg.contract(d.data_ptr())
        assert err.value.status == 1


def test_multilevel_to_one_percent(mm, orc, torch_cuda):
    g = mm.Graph.rgg(1 << 15, 13.0, seed=7)
    seeds = orc.rand_seeds(12345, 256)
    levels = mm.multilevel(g, 9, seeds, target=0.01, device=0)
    sizes = [lv["n"] for lv in levels]
    assert sizes[0] == g.n and sizes[-1] <= 0.01 * g.n + 1
    assert all(a > b for a, b in zip(sizes, sizes[1:]))
    for lv in levels[:-1]:
        assert lv["valid"] and lv["maximal"]
