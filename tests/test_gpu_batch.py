"""Batched matching (mm_graph_set_batch / mm_match_batch): many independent
graphs of different kinds and sizes matched in one launch must give, graph by
graph, the oracle's matching of that graph alone with the same seeds (the
reference's per-call result), and each graph's own round count."""
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


def _batch(mm, rng, count):
    graphs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(40), np.log(6000))))
        kind = i % 4
        if kind == 0:
            wd = max(1, int(np.sqrt(n)))
            graphs.append(mm.Graph.grid(wd, max(1, n // wd)).with_pair_weights(i))
        elif kind == 1:
            graphs.append(mm.Graph.rgg(n, 13.0, seed=i + 1))
        elif kind == 2:
            graphs.append(mm.Graph.er(max(n, 2), 8.0, seed=i + 1))
        else:
            graphs.append(mm.Graph.rmat(max(4, int(np.log2(n))), 8, seed=i + 1))
    return graphs


@pytest.mark.parametrize("type_", [6, 7, 8, 9])
def test_batch_equals_separate_matchings(mm, orc, torch_cuda, type_):
    rng = np.random.default_rng(11)
    graphs = _batch(mm, rng, 48)
    u, off = mm.Graph.union(graphs)
    seeds = orc.rand_seeds(12345, 256)
    with mm.DeviceGraph(u, device=0) as dg:
        dg.set_batch(off)
        out = torch_cuda.empty(u.n, dtype=torch_cuda.int32, device="cuda")
        rounds = dg.match_batch(type_, seeds, out.data_ptr())
        got = out.cpu().numpy()
    for i, g in enumerate(graphs):
        want, want_rounds, _ = orc.match(g, type_, seeds, BARRIER)
        assert rounds[i] == want_rounds, (i, g.name)
        assert np.array_equal(got[off[i]:off[i + 1]], want), (i, g.name)


def test_batch_with_empty_and_adversarial_graphs(mm, orc, torch_cuda):
    rng = np.random.default_rng(3)
    graphs = [random_graph(np.random.default_rng(s), 30 + 17 * s, 4.0, symmetric=s % 2 == 0, gaps=s % 3 == 0)
              for s in range(8)]
    graphs.insert(3, mm.Graph.grid(1, 1))
    u, off = mm.Graph.union(graphs)
    seeds = orc.rand_seeds(7, 256)
    with mm.DeviceGraph(u, device=0) as dg:
        dg.set_batch(off)
        for t in (7, 9):
            out = torch_cuda.empty(u.n, dtype=torch_cuda.int32, device="cuda")
            rounds = dg.match_batch(t, seeds, out.data_ptr())
            got = out.cpu().numpy()
            for i, g in enumerate(graphs):
                want, want_rounds, _ = orc.match(g, t, seeds, BARRIER)
                assert rounds[i] == want_rounds and np.array_equal(got[off[i]:off[i + 1]], want), (t, i)


def test_batch_rejects_crossing_edges(mm, torch_cuda):
    g = mm.Graph.grid(4, 4)
    with mm.DeviceGraph(g, device=0) as dg:
        with pytest.raises(mm.MatchError) as err:
            dg.set_batch(np.array([0, 8, 16], dtype=np.int32))  # grid rows 0-1 and 2-3 share edges
        assert err.value.status == 2
        with pytest.raises(mm.MatchError):
            dg.set_batch(np.array([0, 9, 8, 16], dtype=np.int32))
