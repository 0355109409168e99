"""GPU parity tests: the CUDA paths (push, the product default, and the
reference-structured pull family) against the golden fixtures made from the
reference's own code and against the oracle, bit for bit, through the C ABI."""
from __future__ import annotations

import ctypes
import hashlib

import numpy as np
import pytest

from graphs_small import SmallGraph, random_graph

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def gpu_match(mm, torch, g, type_, seeds, barrier=BARRIER, path=0, dg=None):
    own = dg is None
    if own:
        dg = mm.DeviceGraph(g, device=0)
    try:
        out = torch.full((max(g.n, 1),), -7, dtype=torch.int32, device="cuda")
        rounds = dg.match_device(type_, seeds, out.data_ptr(), barrier=barrier, path=path)
        torch.cuda.synchronize()
        return out[: g.n].cpu().numpy(), rounds
    finally:
        if own:
            dg.close()


PATHS = [("push", 2), ("pull", 1)]


@pytest.mark.parametrize("path_name,path", PATHS)
def test_golden_fixtures(mm, orc, golden, torch_cuda, path_name, path):
    graphs = {}
    devs = {}
    n_checked = 0
    try:
        for c in golden.cases():
            name = c["graph"]
            if name not in graphs:
                graphs[name] = golden.graph(mm, name)
                devs[name] = mm.DeviceGraph(graphs[name], device=0)
            seeds = orc.rand_seeds(c["seed"], 256)
            got, rounds = gpu_match(mm, torch_cuda, graphs[name], c["type"], seeds, c["barrier"], path,
                                    dg=devs[name])
            assert rounds == c["rounds"], c["key"]
            want = golden.match(c["key"])
            if want is not None:
                assert np.array_equal(got, want), (c["key"], int((got != want).sum()))
            assert hashlib.sha256(got.astype(np.int32).tobytes()).hexdigest() == c["sha256"], c["key"]
            n_checked += 1
    finally:
        for d in devs.values():
            d.close()
    assert n_checked > 300


@pytest.mark.parametrize("path_name,path", PATHS)
def test_generated_graphs_match_oracle(mm, orc, torch_cuda, path_name, path):
    graphs = [mm.Graph.grid(512, 512), mm.Graph.rgg(1 << 16, 13.0, seed=7), mm.Graph.rmat(15, 16, seed=1),
              mm.Graph.er(1 << 15, 8.0, seed=1), mm.Graph.rgg(1 << 14, 13.0, seed=3, unit=True)]
    for g in graphs:
        with mm.DeviceGraph(g, device=0) as dg:
            for seed in (1, 12345):
                seeds = orc.rand_seeds(seed, 256)
                for t in mm.TYPES:
                    want, rounds, _ = orc.match(g, t, seeds, BARRIER)
                    got, got_rounds = gpu_match(mm, torch_cuda, g, t, seeds, BARRIER, path, dg=dg)
                    assert got_rounds == rounds, (g.name, t, seed)
                    assert np.array_equal(got, want), (g.name, t, seed, int((got != want).sum()))


@pytest.mark.parametrize("path_name,path", PATHS)
def test_adversarial_graphs_match_oracle(mm, orc, torch_cuda, path_name, path):
    rng = np.random.default_rng(31337)
    for it in range(60):
        n = int(rng.integers(1, 300))
        g = random_graph(rng, n, avg_deg=float(rng.uniform(0.5, 9)), symmetric=bool(rng.random() < 0.6),
                         gaps=bool(rng.random() < 0.3), shuffle_ranges=bool(rng.random() < 0.3),
                         empty_reversed=0.2 if rng.random() < 0.3 else 0.0, dup=0.1, loops=0.1)
        seeds = orc.rand_seeds(int(rng.integers(1, 10000)), 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for barrier in (BARRIER, 0x40000000, 0, 0xFFFFFFFF):
                for t in mm.TYPES:
                    want, rounds, _ = orc.match(g, t, seeds, barrier)
                    got, got_rounds = gpu_match(mm, torch_cuda, g, t, seeds, barrier, path, dg=dg)
                    assert got_rounds == rounds, (it, t, hex(barrier))
                    assert np.array_equal(got, want), (it, t, hex(barrier), int((got != want).sum()))


def test_sorted_lists_match_oracle(mm, orc, torch_cuda):
    """Sorted neighbour lists take the binary-search reverse-key build: duplicates,
    self-loops, one-directional entries, gaps, lists out of vertex order, reversed
    empty ranges, a run of isolated vertices longer than one slot chunk (2048),
    hubs; and one descending pair anywhere sends the graph to the pair-sort build."""
    rng = np.random.default_rng(4242)
    graphs = []
    for it in range(40):
        n = int(rng.integers(1, 400))
        graphs.append(random_graph(rng, n, avg_deg=float(rng.uniform(0.5, 9)), symmetric=bool(rng.random() < 0.6),
                                   gaps=bool(rng.random() < 0.3), shuffle_ranges=bool(rng.random() < 0.3),
                                   empty_reversed=0.2 if rng.random() < 0.3 else 0.0, dup=0.1, loops=0.1,
                                   sort_lists=True))
    # sorted symmetric graph with two hubs and 5000 isolated vertices (ids 2000..6999)
    # inside one slot chunk
    n = 9000
    active = np.concatenate([np.arange(2, 2000), np.arange(7000, n)])
    lists = [[] for _ in range(n)]
    for h in (0, 1):
        for v in active[h::1 + h]:
            lists[h].append(int(v))
            lists[int(v)].append(h)
    for _ in range(8000):
        u, v = int(rng.choice(active)), int(rng.choice(active))
        if u != v:
            lists[u].append(v)
            lists[v].append(u)
    ranges, nbrs = [], []
    for v in range(n):
        b = len(nbrs)
        nbrs += sorted(lists[v])
        ranges.append((b, len(nbrs)))
    nbrs = np.array(nbrs, np.int32)
    wts = (rng.integers(1, 6, len(nbrs)) / 4).astype(np.float32)
    graphs.append(SmallGraph(n, np.array(ranges), nbrs, wts))
    # the same graph with one list's last two entries swapped (unsorted -> pair sort)
    nb2 = nbrs.copy()
    b, e = ranges[1]
    nb2[e - 2], nb2[e - 1] = nb2[e - 1], nb2[e - 2]
    graphs.append(SmallGraph(n, np.array(ranges), nb2, wts))
    for gi, g in enumerate(graphs):
        seeds = orc.rand_seeds(gi + 1, 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for t in mm.TYPES:
                want, rounds, _ = orc.match(g, t, seeds, BARRIER)
                got, got_rounds = gpu_match(mm, torch_cuda, g, t, seeds, BARRIER, 2, dg=dg)
                assert got_rounds == rounds and np.array_equal(got, want), (gi, t)


def test_long_lists_and_hubs_match_oracle(mm, orc, torch_cuda):
    """Stars and cliques push lists past the block-scan threshold (1024)."""
    n = 6000
    lists = [[] for _ in range(n)]
    for hub in (0, 1, 2):
        for v in range(3, n, 1 + hub):
            lists[hub].append(v)
            lists[v].append(hub)
    for u in range(3000, 3060):
        for v in range(3000, 3060):
            if u != v:
                lists[u].append(v)
    rng = np.random.default_rng(5)
    ranges, nbrs, wts = [], [], []
    for v in range(n):
        b = len(nbrs)
        nbrs += lists[v]
        ranges.append((b, len(nbrs)))
    nbrs = np.array(nbrs, np.int32)
    wts = (rng.integers(1, 6, len(nbrs)) / 4).astype(np.float32)
    g = SmallGraph(n, np.array(ranges), nbrs, wts)
    with mm.DeviceGraph(g, device=0) as dg:
        for seed in (2, 3):
            seeds = orc.rand_seeds(seed, 256)
            for t in mm.TYPES:
                want, rounds, _ = orc.match(g, t, seeds, BARRIER)
                for path in (2, 1):
                    got, got_rounds = gpu_match(mm, torch_cuda, g, t, seeds, BARRIER, path, dg=dg)
                    assert got_rounds == rounds and np.array_equal(got, want), (t, seed, path)


def test_degree_class_boundaries_non_contiguous(mm, orc, torch_cuda):
    """Lists of exactly 32/33/2048/2049/4096/4097 entries (the scan's class and
    chunk edges), stored out of vertex order with gaps between lists."""
    rng = np.random.default_rng(17)
    n = 9000
    lists = [[] for _ in range(n)]
    hubs = {0: 32, 1: 33, 2: 2048, 3: 2049, 4: 4096, 5: 4097, 6: 6144}
    for h, d in hubs.items():
        for v in rng.choice(np.arange(10, n), size=d, replace=False):
            lists[h].append(int(v))
            lists[int(v)].append(h)
    for _ in range(20000):
        u, v = int(rng.integers(10, n)), int(rng.integers(10, n))
        if u != v:
            lists[u].append(v)
            lists[v].append(u)
    order = rng.permutation(n)
    ranges = np.zeros((n, 2), np.int64)
    nbrs = []
    for v in order:
        nbrs += [int(x) for x in rng.integers(0, n, int(rng.integers(0, 3)))]  # gap
        b = len(nbrs)
        nbrs += lists[v]
        ranges[v] = (b, len(nbrs))
    nbrs = np.array(nbrs, np.int32)
    wts = (rng.integers(1, 5, len(nbrs)) / 4).astype(np.float32)
    g = SmallGraph(n, ranges, nbrs, wts)
    with mm.DeviceGraph(g, device=0) as dg:
        for seed in (1, 2, 3):
            seeds = orc.rand_seeds(seed, 256)
            for t in mm.TYPES:
                want, rounds, _ = orc.match(g, t, seeds, BARRIER)
                got, got_rounds = gpu_match(mm, torch_cuda, g, t, seeds, BARRIER, 2, dg=dg)
                assert got_rounds == rounds and np.array_equal(got, want), (t, seed)


@pytest.mark.parametrize("path", [2, 1])
def test_round_counters_match_oracle(mm, orc, torch_cuda, path):
    cols = [(0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (6, 6), (7, 7)]  # (mm, oracle) column pairs
    for g in (mm.Graph.rmat(14, 16, seed=2), mm.Graph.rgg(1 << 14, 13.0, seed=7), mm.Graph.grid(128, 128)):
        seeds = orc.rand_seeds(12345, 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for t in mm.TYPES:
                _, rounds, ost = orc.match(g, t, seeds, BARRIER)
                out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
                r, st = dg.stats(t, seeds, out.data_ptr(), path=path)
                assert r == rounds
                for a, b in cols:
                    assert np.array_equal(st[:, a], ost[:, b]), (g.name, t, a)


def test_host_output_api_and_repeat_calls(mm, orc, torch_cuda):
    g = mm.Graph.rgg(1 << 15, 13.0, seed=11)
    seeds = orc.rand_seeds(99, 256)
    want, rounds, _ = orc.match(g, 9, seeds, BARRIER)
    with mm.DeviceGraph(g, device=0) as dg:
        dg.prepare(9)
        for _ in range(3):
            got, r = dg.match(9, seeds)
            assert r == rounds and np.array_equal(got, want)
        # another type on the same object, then back
        want7, r7, _ = orc.match(g, 7, seeds, BARRIER)
        got7, rr7 = dg.match(7, seeds)
        assert rr7 == r7 and np.array_equal(got7, want7)
        got, r = dg.match(9, seeds)
        assert r == rounds and np.array_equal(got, want)


def test_edge_cases(mm, orc, torch_cuda):
    seeds = orc.rand_seeds(1, 256)
    # no vertices: the reference still runs one (maximal) or twenty (fixed) rounds
    g0 = SmallGraph(0, np.zeros((0, 2)), np.zeros(0), np.zeros(0))
    with mm.DeviceGraph(g0, device=0) as dg:
        assert dg.match(7, seeds)[1] == 1
        assert dg.match(8, seeds)[1] == 20
    # isolated vertices only: every vertex dies once it turns blue
    g1 = SmallGraph(50, np.zeros((50, 2)), np.zeros(0), np.zeros(0))
    for t in mm.TYPES:
        want, rounds, _ = orc.match(g1, t, seeds, BARRIER)
        got, r = gpu_match(mm, torch_cuda, g1, t, seeds)
        assert r == rounds and np.array_equal(got, want)
    # barrier 0: nobody is ever blue, the maximal loop hits its 255-round cap
    g2 = mm.Graph.grid(10, 10)
    for t in mm.TYPES:
        want, rounds, _ = orc.match(g2, t, seeds, 0)
        got, r = gpu_match(mm, torch_cuda, g2, t, seeds, barrier=0)
        assert r == rounds and np.array_equal(got, want)
        assert rounds == (255 if t in (7, 9) else 20)


def test_isolated_vertices_beside_a_graph(mm, orc, torch_cuda):
    """Vertices without neighbours (resolved at set-up on the symmetric path, a hash
    per vertex and round): 2^20 of them after a random geometric graph, with
    barriers that keep them red for a few rounds, for dozens, and to the cap; and
    seed sequences one short of the rounds the reference draws, which must be an
    error, or exactly enough."""
    seeds = orc.rand_seeds(3, 256)
    base = mm.Graph.rgg(1 << 12, 13.0, seed=3)
    extra = 1 << 20
    r = np.concatenate([np.asarray(base.ranges, np.int64),
                        np.full((extra, 2), base.nnz, np.int64)]).astype(np.int32)
    g = mm.Graph(base.n + extra, r, base.nbrs, base.weights, "rgg-and-isolated")
    with mm.DeviceGraph(g, device=0) as dg:
        for barrier in (BARRIER, 0x10000000, 0x01000000):
            for t in mm.TYPES:
                want, rounds, _ = orc.match(g, t, seeds, barrier)
                got, rr = gpu_match(mm, torch_cuda, g, t, seeds, barrier=barrier, dg=dg)
                assert rr == rounds and np.array_equal(got, want), (hex(barrier), t, rr, rounds)
        want, rounds, _ = orc.match(g, 7, seeds, 0x10000000)
        assert rounds < 255
        with pytest.raises(mm.MatchError) as e:
            dg.match(7, seeds[: rounds - 1], barrier=0x10000000)
        assert e.value.status == 6
        got, rr = dg.match(7, seeds[:rounds], barrier=0x10000000)
        assert rr == rounds and np.array_equal(got, want)


def test_errors_are_statuses(mm, orc, torch_cuda):
    seeds = orc.rand_seeds(1, 256)
    bad_id = SmallGraph(3, np.array([[0, 2], [2, 3], [3, 3]]), np.array([1, 5, 0]), None)
    with pytest.raises(mm.MatchError) as e:
        mm.DeviceGraph(bad_id, device=0)
    assert e.value.status == 2
    bad_range = SmallGraph(2, np.array([[0, 4], [1, 1]]), np.array([1, 0]), None)
    with pytest.raises(mm.MatchError) as e:
        mm.DeviceGraph(bad_range, device=0)
    assert e.value.status == 2
    g = mm.Graph.grid(64, 64)
    with mm.DeviceGraph(g, device=0) as dg:
        with pytest.raises(mm.MatchError) as e:
            dg.match(7, seeds[:3])  # the maximal loop needs more rounds than seeds
        assert e.value.status == 6
        with pytest.raises(mm.MatchError) as e:
            dg.match(5, seeds)
        assert e.value.status == 1
        # the object stays usable after errors
        want, rounds, _ = orc.match(g, 7, seeds, BARRIER)
        got, r = dg.match(7, seeds)
        assert r == rounds and np.array_equal(got, want)


def test_rgg_config_full_size(mm, orc, torch_cuda):
    """The random geometric graph at full size: 2^20 vertices, average degree 13, weighted, seed 7."""
    g = mm.Graph.rgg(1 << 20, 13.0, seed=7)
    seeds = orc.rand_seeds(12345, 256)
    with mm.DeviceGraph(g, device=0) as dg:
        for t in (8, 9):
            want, rounds, _ = orc.match(g, t, seeds, BARRIER)
            got, r = gpu_match(mm, torch_cuda, g, t, seeds, dg=dg)
            assert r == rounds and np.array_equal(got, want)
            if t == 9:
                chk = orc.check(g, got)
                assert chk["valid"] and chk["matchable"] == 0


def test_launch_options_never_change_the_result(mm, orc, torch_cuda):
    """mm_graph_tune changes only the time: every finish-phase divisor (2 tries the
    phase so early that attempts are called off and the resumed round kernel
    carries on; -1 never enters it) and block count gives the oracle's matching."""
    seeds = orc.rand_seeds(12345, 256)
    for g in (mm.Graph.rgg(1 << 14, 13.0, seed=7), mm.Graph.rmat(14, 16, seed=2), mm.Graph.grid(100, 90)):
        with mm.DeviceGraph(g, device=0) as dg:
            for t in (7, 9):
                want, rounds, _ = orc.match(g, t, seeds, BARRIER)
                for d in (-1, 2, 3, 12, 40):
                    for b in (1, 2):
                        dg.tune(d, b)
                        got, r = gpu_match(mm, torch_cuda, g, t, seeds, dg=dg)
                        assert r == rounds and np.array_equal(got, want), (g.name, t, d, b)
            dg.tune(0, 0)
